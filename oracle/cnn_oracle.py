"""TEST INFRASTRUCTURE ONLY -- not part of the product.

FP64 numpy restatement of the learned Richardson-Lucy proposal's layer (the
sparse APR CNN of libapr_b200/csrc/learned.cu), the checker of its forward and
backward kernels.  There is no reference implementation of this network; its
neighbourhood is the one of LibAPR's APRFilter::convolve_pencil
(src/numerics/APRFilter.hpp:766-849: same-level particles, parents one level
coarser, tree means of the level) with a zero boundary, and its tree means are
APRTreeNumerics::fill_tree_mean (src/numerics/APRTreeNumerics.hpp:63-203,
scale factors :97-110) applied channel by channel.

Layout: particle features P x 16 (channels-last), weights W[27][16 out][16 in]
with taps t = (iz * 3 + ix) * 3 + iy at offsets (iz - 1, ix - 1, iy - 1).
`bf16=True` rounds the products' operands (weights, neighbourhood values,
output gradients) to bfloat16 as the tensor cores see them; sums stay FP64.
"""
import numpy as np

C = 16


def bf16(a):
    """Round float values to the nearest bfloat16 (ties to even), as float64."""
    a32 = np.ascontiguousarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


class Geometry:
    """Per-level particle and tree-node coordinates of an APR (oracle Access
    objects for the APR and its tree)."""

    def __init__(self, acc, tree):
        self.acc, self.tree = acc, tree
        self.plev, self.pz, self.px, self.py = acc.particle_coords()
        self.tlev, self.tz, self.tx, self.ty = tree.particle_coords()
        self.P, self.T = acc.P, tree.P
        # parent tree node and weight (scale factor / 8) of every particle and tree node
        self.p_par, self.p_w = self._parents(self.plev, self.pz, self.px, self.py)
        self.t_par, self.t_w = self._parents(self.tlev, self.tz, self.tx, self.ty)

    def dims(self, l):
        a = self.acc
        return a.z_num[l], a.x_num[l], a.y_num[l]

    def _parents(self, lev, z, x, y):
        t = self.tree
        par = np.full(len(lev), -1, np.int64)
        w = np.zeros(len(lev))
        index = {}
        for k in range(self.T):
            index[(int(self.tlev[k]), int(self.tz[k]), int(self.tx[k]), int(self.ty[k]))] = k
        for i in range(len(lev)):
            l = int(lev[i]) - 1
            if l < t.l_min:
                continue
            zp, xp, yp = int(z[i]) // 2, int(x[i]) // 2, int(y[i]) // 2
            k = index.get((l, zp, xp, yp))
            if k is None:
                continue
            zt, xt, yt = t.z_num[l], t.x_num[l], t.y_num[l]
            zc, xc, yc = self.acc.z_num[l + 1], self.acc.x_num[l + 1], self.acc.y_num[l + 1]
            sxz = float(((2 * xt != xc) and (xp == xt - 1)) + ((2 * zt != zc) and (zp == zt - 1))) * 2
            if sxz == 0:
                sxz = 1.0
            syxz = sxz * 2 if 2 * yt != yc else sxz
            par[i] = k
            w[i] = (syxz if yp == yt - 1 else sxz) / 8.0
        return par, w


def tree_means(geo, H):
    """Multi-channel fill_tree_mean: tree levels fine to coarse."""
    HT = np.zeros((geo.T, H.shape[1]))
    for l in range(geo.tree.l_max, geo.tree.l_min - 1, -1):
        c = l + 1
        m = (geo.plev == c) & (geo.p_par >= 0)
        np.add.at(HT, geo.p_par[m], geo.p_w[m][:, None] * H[m])
        m = (geo.tlev == c) & (geo.t_par >= 0)
        np.add.at(HT, geo.t_par[m], geo.t_w[m][:, None] * HT[m])
    return HT


def level_image(geo, l, H, HT):
    """Neighbourhood image of level l, zero-padded by one cell: (z+2, x+2, y+2, C)."""
    zn, xn, yn = geo.dims(l)
    D = np.zeros((zn + 2, xn + 2, yn + 2, H.shape[1]))
    m = geo.plev == l
    D[geo.pz[m] + 1, geo.px[m] + 1, geo.py[m] + 1] = H[m]
    if l > geo.acc.l_min:
        m = np.nonzero(geo.plev == l - 1)[0]
        for dz in (0, 1):
            for dx in (0, 1):
                for dy in (0, 1):
                    z = 2 * geo.pz[m] + dz
                    x = 2 * geo.px[m] + dx
                    y = np.minimum(2 * geo.py[m] + dy, yn - 1)
                    ok = (z < zn) & (x < xn)
                    D[z[ok] + 1, x[ok] + 1, y[ok] + 1] = H[m[ok]]
    if l <= geo.tree.l_max:
        m = geo.tlev == l
        D[geo.tz[m] + 1, geo.tx[m] + 1, geo.ty[m] + 1] = HT[m]
    return D


TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def layer_forward(geo, H, W, b, relu, round_bf16=False):
    HT = tree_means(geo, H)
    out = np.zeros((geo.P, W.shape[1]))
    Wm = bf16(W) if round_bf16 else np.asarray(W, np.float64)
    for l in range(geo.acc.l_min, geo.acc.l_max + 1):
        m = np.nonzero(geo.plev == l)[0]
        if len(m) == 0:
            continue
        D = level_image(geo, l, H, HT)
        if round_bf16:
            D = bf16(D)
        acc = np.zeros((len(m), W.shape[1]))
        for t, (dz, dx, dy) in enumerate(TAPS):
            g = D[geo.pz[m] + 1 + dz, geo.px[m] + 1 + dx, geo.py[m] + 1 + dy]
            acc += g @ Wm[t].T
        out[m] = acc + b[None, :]
    return np.maximum(out, 0.0) if relu else out


def layer_backward(geo, H, W, out, g_out, relu, round_bf16=False):
    """(g_in, dW, db) of one layer."""
    HT = tree_means(geo, H)
    gp = g_out * (out > 0) if relu else np.array(g_out, np.float64)
    Wm = bf16(W) if round_bf16 else np.asarray(W, np.float64)
    gpm = bf16(gp) if round_bf16 else gp
    dW = np.zeros_like(np.asarray(W, np.float64))
    db = gp.sum(axis=0)
    g_in = np.zeros_like(np.asarray(H, np.float64))
    g_tree = np.zeros((geo.T, H.shape[1]))
    for l in range(geo.acc.l_min, geo.acc.l_max + 1):
        m = np.nonzero(geo.plev == l)[0]
        if len(m) == 0:
            continue
        zn, xn, yn = geo.dims(l)
        D = level_image(geo, l, H, HT)
        if round_bf16:
            D = bf16(D)
        dD = np.zeros((zn + 2, xn + 2, yn + 2, H.shape[1]))
        for t, (dz, dx, dy) in enumerate(TAPS):
            zi, xi, yi = geo.pz[m] + 1 + dz, geo.px[m] + 1 + dx, geo.py[m] + 1 + dy
            dW[t] += gpm[m].T @ D[zi, xi, yi]
            np.add.at(dD, (zi, xi, yi), gpm[m] @ Wm[t])
        dD = dD[1:-1, 1:-1, 1:-1]
        g_in[m] += dD[geo.pz[m], geo.px[m], geo.py[m]]
        if l > geo.acc.l_min:
            mp = np.nonzero(geo.plev == l - 1)[0]
            for dz in (0, 1):
                for dx in (0, 1):
                    z = 2 * geo.pz[mp] + dz
                    x = 2 * geo.px[mp] + dx
                    ok = (z < zn) & (x < xn)
                    y0 = 2 * geo.py[mp]
                    y1 = np.minimum(y0 + 1, yn - 1)
                    g_in[mp[ok]] += dD[z[ok], x[ok], y0[ok]]
                    two = ok & (y1 != y0)
                    g_in[mp[two]] += dD[z[two], x[two], y1[two]]
        if l <= geo.tree.l_max:
            mt = geo.tlev == l
            g_tree[mt] += dD[geo.tz[mt], geo.tx[mt], geo.ty[mt]]
    # tree means transposed, coarse to fine
    for l in range(geo.tree.l_min, geo.tree.l_max + 1):
        c = l + 1
        m = (geo.tlev == c) & (geo.t_par >= 0)
        g_tree[m] += geo.t_w[m][:, None] * g_tree[geo.t_par[m]]
        m = (geo.plev == c) & (geo.p_par >= 0)
        g_in[m] += geo.p_w[m][:, None] * g_tree[geo.p_par[m]]
    return g_in, dW, db
