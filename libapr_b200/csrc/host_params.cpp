// Host-side constants for the GPU pipeline.  The reference evaluates these
// expressions with float variables but unqualified libm calls on float
// arguments, which resolve to the double-precision functions; every such step
// is written here as an explicit double evaluation followed by the float
// store the reference performs.
#include "host_params.hpp"

#include <cmath>
#include <cstring>

namespace aprb {

namespace {

float impulse_resp(float k, float rho, float omg) {  // ComputeGradient.hpp:206-211
    float ak = std::fabs(k);
    return (float)((std::pow((double)rho, (double)ak) * std::sin((double)((ak + 1) * omg))) / std::sin((double)omg));
}

float impulse_resp_back(float k, float rho, float omg, float gamma, float c0) {  // :213-218
    float ak = std::fabs(k);
    double p2 = std::pow((double)rho, 2.0);
    double den = std::pow(1.0 - 2.0 * (double)rho * std::cos((double)omg) + p2, 2.0);
    return (float)((double)c0 * std::pow((double)rho, (double)ak) *
                   (std::cos((double)(omg * ak)) + (double)gamma * std::sin((double)(omg * ak))) * (1.0 / den));
}

double powr(double num, double p) { return std::round(std::pow(num, p)); }

}  // namespace

IIRCoef iir_coefficients(float lambda, int dim) {
    const float tol = 0.0001f;
    IIRCoef c;
    float xi = (float)((double)(1.0f - 96.0f * lambda) +
                       (double)(24.0f * lambda) * std::sqrt((double)(3.0f + 144.0f * lambda)));
    double inner = (double)(48.0f * lambda) + (double)(24.0f * lambda) * std::sqrt((double)(3.0f + 144.0f * lambda));
    float rho = (float)(((double)(24.0f * lambda - 1.0f) - std::sqrt((double)xi)) / (double)(24.0f * lambda) *
                        std::sqrt((double)(1.0f / xi) * inner));
    float omg = (float)std::atan(std::sqrt((double)((1.0f / xi) * (144.0f * lambda - 1.0f))));
    double p2 = std::pow((double)rho, 2.0);
    double cw = std::cos((double)omg);
    float c0 = (float)((1.0 + p2) / (1.0 - p2) * (1.0 - (double)(2.0f * rho) * cw + p2) /
                       (1.0 + (double)(2.0f * rho) * cw + p2));
    float gamma = (float)((1.0 - p2) / (1.0 + p2) * (1.0 / std::tan((double)omg)));
    c.b1 = (float)((double)(2.0f * rho) * cw);
    c.b2 = (float)(-std::pow((double)rho, 2.0));
    const int k0 = (int)std::ceil(std::fabs(std::log((double)tol) / std::log((double)rho)));
    c.k0 = k0;
    c.minLen = k0 < dim ? k0 : dim;
    c.norm = (float)std::pow(1.0 - 2.0 * (double)rho * cw + p2, 2.0);
    if (k0 < 2) return c;
    std::vector<float> irf(k0 + 3), irb(k0 + 3);
    for (int k = 0; k < k0 + 3; ++k) irf[k] = impulse_resp((float)k, rho, omg);
    for (int k = 0; k < k0 + 3; ++k) irb[k] = impulse_resp_back((float)k, rho, omg, gamma, c0);
    std::vector<float> b1(k0, 0.0f), b2(k0, 0.0f), b3(k0, 0.0f), b4(k0, 0.0f);
    const int m = c.minLen;
    b1[1] = irf[0];
    for (int k = 0; k < k0; ++k) b1[k] += irf[k + 1];
    for (int k = m; k < k0; ++k) b1[m - 1] += b1[k];
    for (int k = 0; k < k0; ++k) b2[k] = irf[k];
    for (int k = m; k < k0; ++k) b2[m - 1] += b2[k];
    b3[0] = irb[1];
    for (int k = 0; k < k0 - 1; ++k) b3[k + 1] += irb[k] + irb[k + 2];
    for (int k = m; k < k0; ++k) b3[m - 1] += b3[k];
    b4[0] = irb[0];
    for (int k = 1; k < k0; ++k) b4[k] += 2 * irb[k];
    for (int k = m; k < k0; ++k) b4[m - 1] += b4[k];
    c.bc1.assign(b1.begin(), b1.begin() + m);
    c.bc2.assign(b2.begin(), b2.begin() + m);
    c.bc3.assign(b3.begin(), b3.begin() + m);
    c.bc4.assign(b4.begin(), b4.begin() + m);
    return c;
}

LisWindow lis_window(const aprb_params &p, int yd, int xd, int zd) {
    static const double r3[6] = {12.8214, 26.1256, 40.2795, 23.3692, 36.2061, 27.0385};
    static const double r2[6] = {13.2421, 28.7069, 52.0385, 24.4272, 34.9565, 21.1891};
    static const double r1[6] = {13.9040, 31.2843, 57.4037, 30.3767, 45.9930, 29.0890};
    static const int w1[6] = {1, 1, 1, 2, 2, 3};
    static const int w2[6] = {2, 3, 4, 4, 5, 6};
    LisWindow w;
    float fi = (float)(std::round((double)(p.psfx / p.dx)) - 1);
    int psf_ind = (int)(fi > 0.0f ? fi : 0.0f);
    if (psf_ind > 5) psf_ind = 5;
    int win_val = w1[psf_ind] > w2[psf_ind] ? w1[psf_ind] : w2[psf_ind];
    int dims[3] = {yd, xd, zd};
    for (int a = 0; a < 3; ++a) {
        w.active[a] = dims[a] > win_val;
        w.win1[a] = w.active[a] ? w1[psf_ind] : 0;
        w.win2[a] = w.active[a] ? w2[psf_ind] : 0;
        w.n_active += w.active[a];
    }
    w.rescale = (float)(w.n_active == 3 ? r3[psf_ind] : w.n_active == 2 ? r2[psf_ind] : r1[psf_ind]);
    return w;
}

static uint64_t xz_linear(Geom &g) {
    uint64_t counter = 1;
    std::memset(g.level_xz, 0, sizeof(g.level_xz));
    g.level_xz[0] = 1;
    for (int i = 0; i <= g.l_max; ++i) {
        counter += (uint64_t)g.x_num[i] * (uint64_t)g.z_num[i];
        g.level_xz[i + 1] = counter;
    }
    return counter;
}

uint64_t apr_geometry(int y, int x, int z, Geom &g) {
    std::memset(&g, 0, sizeof(g));
    int max_dim = std::max(std::max(x, y), z);
    int lm = std::max(1, (int)std::ceil(std::log2((double)max_dim)));
    g.l_min = 1;
    g.l_max = lm;
    for (int l = g.l_min; l <= g.l_max; ++l) {
        double cell = powr(2, lm - l);
        g.y_num[l] = (int)std::ceil((double)(uint64_t)y / cell);
        g.x_num[l] = (int)std::ceil((double)(uint64_t)x / cell);
        g.z_num[l] = (int)std::ceil((double)(uint64_t)z / cell);
    }
    return xz_linear(g);
}

uint64_t tree_geometry(int y, int x, int z, Geom &g) {
    std::memset(&g, 0, sizeof(g));
    int max_dim = std::max(std::max(x, y), z);
    int lm = (int)std::ceil(std::log2((double)max_dim));
    g.l_min = 0;
    g.l_max = std::max(lm - 1, 0);
    for (int l = g.l_min; l <= g.l_max; ++l) {
        double cell = powr(2, g.l_max - l + 1);
        g.y_num[l] = (int)std::ceil((double)(uint64_t)y / cell);
        g.x_num[l] = (int)std::ceil((double)(uint64_t)x / cell);
        g.z_num[l] = (int)std::ceil((double)(uint64_t)z / cell);
    }
    return xz_linear(g);
}

template <typename T>
std::vector<T> downsampled_stencils(const T *in, int ks, int nlevels, bool normalize, std::vector<int> &sides) {
    if (nlevels < 1) nlevels = 1;
    const int n0 = ks * ks * ks;
    std::vector<T> out(in, in + n0);
    if (normalize) {  // PixelData::normalize (PixelData.hpp:771-778): the sum is a float
        float s = 0.0f;
        for (int i = 0; i < n0; ++i) s = (float)(s + out[i]);
        if (std::fabs(s) > 1e-6 && s != 1.0f)
            for (int i = 0; i < n0; ++i) out[i] = out[i] / s;
    }
    sides.assign(1, ks);
    for (int d = 1; d < nlevels; ++d) {  // downsample_stencil (APRStencil.hpp:13-77)
        const int step = (int)std::pow(2.0f, (float)d);
        const int factor = (int)std::pow((float)step, 3.0f);
        int nd = 2 * (((ks - 1) / 2 + step - 1) / step) + 1;
        if (nd < 3) nd = 3;
        std::vector<T> o((size_t)nd * nd * nd, T(0));
        const int off = (nd / 2) * step - ks / 2;
        for (int iz = 0; iz < ks; ++iz)
            for (int ix = 0; ix < ks; ++ix)
                for (int iy = 0; iy < ks; ++iy)
                    for (int dz = 0; dz < nd; ++dz) {
                        int zs = std::max(dz * step, off + iz), ze = std::min(dz * step + step, off + iz + step);
                        float oz = (float)std::max(ze - zs, 0);
                        for (int dx = 0; dx < nd; ++dx) {
                            int xs = std::max(dx * step, off + ix), xe = std::min(dx * step + step, off + ix + step);
                            float ox = (float)std::max(xe - xs, 0);
                            for (int dy = 0; dy < nd; ++dy) {
                                int ys = std::max(dy * step, off + iy), ye = std::min(dy * step + step, off + iy + step);
                                float oy = (float)std::max(ye - ys, 0);
                                float ov = ox * oy * oz;
                                o[((size_t)dz * nd + dx) * nd + dy] += ov * in[((size_t)iz * ks + ix) * ks + iy];
                            }
                        }
                    }
        float sum = 0;  // a float in the reference for every stencil type
        for (auto &v : o) {
            v /= factor;
            sum = (float)(sum + v);
        }
        if (normalize) {
            float nf = 1.0f / sum;
            for (auto &v : o) v *= nf;
        }
        out.insert(out.end(), o.begin(), o.end());
        sides.push_back(nd);
    }
    return out;
}

template std::vector<float> downsampled_stencils<float>(const float *, int, int, bool, std::vector<int> &);
template std::vector<double> downsampled_stencils<double>(const double *, int, int, bool, std::vector<int> &);

}  // namespace aprb
