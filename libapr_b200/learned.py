"""Learned Richardson-Lucy proposal (no counterpart in the reference).

A sparse CNN on APR particles -- 4 layers of per-level 3x3x3 stencils with
channels 3 -> 16 -> 16 -> 16 -> 1, bfloat16 operands on the tensor cores with
float accumulation (libapr_b200/csrc/learned.cu) -- predicts the
log-multiplicative update of ten Richardson-Lucy iterations from the current
estimate u, the RL ratio d / conv(psf_flipped, u) and the data d.  Plain RL
resumes from the proposal; the proposal is rejected when RL's Poisson
data-fit objective rises.

Every compute step runs in the library's own kernels: the layer forward and
backward passes, the features, the loss and Adam.  torch holds the device
buffers.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import check, lib

CH = 16
TAPS = 27
N_LAYERS = 4
REAL_IN = 3  # real input channels of the first layer
WEIGHTS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "rl_proposal_cnn.npz")


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s(stream):
    return None if stream is None else C.c_void_p(stream.cuda_stream)


class ProposalCNN:
    """Weights W[layer][27][16 out][16 in], biases b[layer][16], on the GPU."""

    def __init__(self, seed=0, device="cuda"):
        import torch
        g = torch.Generator().manual_seed(seed)
        self.W = torch.zeros(N_LAYERS, TAPS, CH, CH)
        self.b = torch.zeros(N_LAYERS, CH)
        for k in range(N_LAYERS):
            fan_in = TAPS * (REAL_IN if k == 0 else CH)
            std = (2.0 / fan_in) ** 0.5 * (0.1 if k == N_LAYERS - 1 else 1.0)
            self.W[k] = torch.randn(TAPS, CH, CH, generator=g) * std
        self.W_mask = torch.ones_like(self.W)
        self.b_mask = torch.ones_like(self.b)
        self.W_mask[0, :, :, REAL_IN:] = 0  # padded input channels
        self.W_mask[N_LAYERS - 1, :, 1:, :] = 0  # one output channel
        self.b_mask[N_LAYERS - 1, 1:] = 0
        self.W = (self.W * self.W_mask).to(device).contiguous()
        self.b = (self.b * self.b_mask).to(device).contiguous()
        self.W_mask = self.W_mask.to(device).contiguous()
        self.b_mask = self.b_mask.to(device).contiguous()
        self.mW = torch.zeros_like(self.W)
        self.vW = torch.zeros_like(self.W)
        self.mb = torch.zeros_like(self.b)
        self.vb = torch.zeros_like(self.b)
        self.step_count = 0

    # ------------------------------------------------------------------ io
    def save(self, path=WEIGHTS_FILE):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, W=self.W.cpu().numpy(), b=self.b.cpu().numpy())

    @classmethod
    def load(cls, path=WEIGHTS_FILE, device="cuda"):
        import torch
        d = np.load(path)
        net = cls(device=device)
        net.W = torch.from_numpy(d["W"]).to(device).contiguous()
        net.b = torch.from_numpy(d["b"]).to(device).contiguous()
        return net

    # ------------------------------------------------------------------ passes
    def forward(self, apr, feat, stream=None):
        """feat: P x 16 float CUDA tensor.  Returns the activations of every
        layer (the input first); the prediction is channel 0 of the last."""
        import torch
        acts = [feat]
        x = feat
        for k in range(N_LAYERS):
            y = torch.empty_like(x)
            check(lib().aprb_cnn_layer_forward_device(apr._h, _p(x), _p(self.W[k]), _p(self.b[k]),
                                                      int(k < N_LAYERS - 1), _p(y), _s(stream)))
            acts.append(y)
            x = y
        return acts

    def backward(self, apr, acts, g_pred, stream=None):
        """Gradients (dW, db) of the loss whose gradient w.r.t. the last
        layer's output is g_pred (P x 16)."""
        import torch
        dW = torch.zeros_like(self.W)
        db = torch.zeros_like(self.b)
        g = g_pred
        for k in range(N_LAYERS - 1, -1, -1):
            g_in = torch.empty_like(acts[k])
            check(lib().aprb_cnn_layer_backward_device(apr._h, _p(acts[k]), _p(self.W[k]), _p(acts[k + 1]), _p(g),
                                                       int(k < N_LAYERS - 1), _p(g_in), _p(dW[k]), _p(db[k]),
                                                       _s(stream)))
            g = g_in
        return dW, db

    def adam_step(self, dW, db, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        for p, gr, m, v, mask in ((self.W, dW, self.mW, self.vW, self.W_mask), (self.b, db, self.mb, self.vb,
                                                                                self.b_mask)):
            check(lib().aprb_cnn_adam_device(_p(p), _p(gr), _p(m), _p(v), _p(mask), p.numel(), lr, beta1, beta2,
                                             eps, self.step_count, _s(stream)))

    # ------------------------------------------------------------------ RL use
    def features(self, apr, raw, u, psf, stream=None):
        """raw: P int16 (uint16 data), u: P float CUDA tensors."""
        import torch
        P = u.numel()
        ratio = torch.empty_like(u)
        st = np.ascontiguousarray(psf, np.float32).ravel()
        ks = int(round(st.size ** (1.0 / 3.0)))
        check(lib().aprb_rl_ratio_device(apr._h, _p(raw), _p(u), _p(ratio), C.c_void_p(st.ctypes.data), ks, 1, 1,
                                         _s(stream)))
        feat = torch.empty(P, CH, device=u.device, dtype=torch.float32)
        check(lib().aprb_cnn_features_device(apr._h, _p(u), _p(ratio), _p(raw), _p(feat), _s(stream)))
        return feat

    def train_step(self, apr, raw, u0, u1, psf, lr=1e-3, stream=None):
        """One Adam step on the pair (u0 = RL iterate i, u1 = iterate i + 10).
        Returns the loss (mean squared log-update error)."""
        import torch
        feat = self.features(apr, raw, u0, psf, stream)
        acts = self.forward(apr, feat, stream)
        g = torch.empty_like(acts[-1])
        loss = torch.zeros(1, dtype=torch.float64, device=u0.device)
        check(lib().aprb_cnn_loss_device(apr._h, _p(acts[-1]), _p(u0), _p(u1), _p(g), _p(loss), _s(stream)))
        dW, db = self.backward(apr, acts, g, stream)
        self.adam_step(dW, db, lr=lr, stream=stream)
        return float(loss.item())

    def loss(self, apr, raw, u0, u1, psf, stream=None):
        import torch
        feat = self.features(apr, raw, u0, psf, stream)
        acts = self.forward(apr, feat, stream)
        g = torch.empty_like(acts[-1])
        loss = torch.zeros(1, dtype=torch.float64, device=u0.device)
        check(lib().aprb_cnn_loss_device(apr._h, _p(acts[-1]), _p(u0), _p(u1), _p(g), _p(loss), _s(stream)))
        return float(loss.item())

    def propose(self, apr, raw, u, psf, stream=None):
        """u <- u * exp(prediction), in place."""
        feat = self.features(apr, raw, u, psf, stream)
        acts = self.forward(apr, feat, stream)
        check(lib().aprb_cnn_apply_device(apr._h, _p(acts[-1]), _p(u), _s(stream)))


DECONV_PARAMS = dict(lambda_=3.0, rel_error=0.1, Ip_th=0.0, sigma_th=50.0, grad_th=10.0)
DECONV_BLOBS = 20000  # per 256 x 1024 x 1024 voxels


def gaussian_psf(sigma=1.2, ks=5):
    """Normalised ks^3 Gaussian PSF (float32, z-x-y order)."""
    g = np.exp(-((np.arange(ks) - ks // 2) ** 2) / (2 * sigma * sigma)).astype(np.float32)
    p = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.float32)
    return (p / p.sum()).astype(np.float32)


def deconvolution_workload(shape, seed, image_type="float", stream=None):
    """The seeded deconvolution workload on the GPU: float ground truth
    (background 50, Gaussian blobs sigma U[1,4], amplitude U[500,5000], 20000
    per 256x1024x1024 voxels) blurred by the normalised 5^3 Gaussian PSF
    (sigma 1.2, replicate border), Poisson noise, uint16; APR with lambda=3,
    E=0.1, Ip_th=0, sigma_th=50, grad_th=10, its tree built.  Returns
    (apr, data particles as an int16 CUDA tensor holding uint16 values, psf,
    number of blobs)."""
    import torch
    import torch.nn.functional as F
    from . import APR, APRConverter, APRParameters, synth_ground_truth_device
    z, x, y = shape
    n = z * x * y
    nb = max(1, int(round(DECONV_BLOBS * n / (256 * 1024 * 1024))))
    gt = torch.empty(shape, dtype=torch.float32, device="cuda")
    synth_ground_truth_device(gt, nb, (1.0, 4.0), (500.0, 5000.0), 50.0, seed=seed, stream=stream)
    psf = gaussian_psf()
    k = torch.from_numpy(psf).cuda().view(1, 1, 5, 5, 5)
    blurred = F.conv3d(F.pad(gt[None, None], (2, 2, 2, 2, 2, 2), mode="replicate"), k)[0, 0]
    del gt
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed + 1)
    noisy = torch.poisson(blurred, generator=gen).clamp_(0, 65535)
    img = noisy.to(torch.int32).to(torch.int16).contiguous()  # low 16 bits: the uint16 value
    del blurred, noisy
    conv = APRConverter(image_type)
    par = APRParameters()
    for key, v in DECONV_PARAMS.items():
        setattr(par, key, v)
    conv.par = par
    apr = APR()
    assert conv.get_apr(apr, img)
    P = apr.total_number_particles()
    raw = torch.empty(max(P, 1), dtype=torch.int16, device="cuda")
    check(lib().aprb_sample_image_device(apr._h, _p(img), _p(raw), _s(stream)))
    del img
    apr.init_tree()
    return apr, raw[:P], psf, nb


def rl_objective(apr, raw, u, psf, stream=None):
    """RL's Poisson data-fit objective sum(k - d log k), k = conv(psf_flipped, u)."""
    st = np.ascontiguousarray(psf, np.float32).ravel()
    ks = int(round(st.size ** (1.0 / 3.0)))
    out = C.c_double()
    check(lib().aprb_rl_objective_device(apr._h, _p(raw), _p(u), C.c_void_p(st.ctypes.data), ks, 1, 1, C.byref(out),
                                         _s(stream)))
    return out.value


def rl_iterations(apr, raw, u, psf, n, resume=True, stream=None):
    """n plain FP32 RL iterations on u in place (stencil down-sampling and
    normalisation on)."""
    st = np.ascontiguousarray(psf, np.float32).ravel()
    ks = int(round(st.size ** (1.0 / 3.0)))
    check(lib().aprb_richardson_lucy_device(apr._h, _p(raw), _p(u), C.c_void_p(st.ctypes.data), ks, int(n), 1, 1,
                                            int(resume), _s(stream)))


class AcceleratedRL:
    """RL with learned proposals, one stage at a time: `warmup` plain
    iterations first, then per stage the network proposes a ten-iteration
    jump, the proposal is kept only when RL's data-fit objective does not rise
    (plain RL is the fallback), and `every` plain iterations follow."""

    def __init__(self, apr, raw, u, psf, net, every=10, warmup=10, stream=None):
        self.apr, self.raw, self.u, self.psf, self.net = apr, raw, u, psf, net
        self.every, self.warmup, self.stream = every, warmup, stream
        self.iterations = 0
        self.tried = self.kept = 0

    def step(self):
        import torch
        if self.iterations == 0:
            rl_iterations(self.apr, self.raw, self.u, self.psf, self.warmup, resume=False, stream=self.stream)
            self.iterations = self.warmup
            return
        before = rl_objective(self.apr, self.raw, self.u, self.psf, self.stream)
        backup = self.u.clone()
        self.net.propose(self.apr, self.raw, self.u, self.psf, self.stream)
        self.tried += 1
        after = rl_objective(self.apr, self.raw, self.u, self.psf, self.stream)
        if not (after <= before) or not bool(torch.isfinite(self.u).all()):
            self.u.copy_(backup)
        else:
            self.kept += 1
        rl_iterations(self.apr, self.raw, self.u, self.psf, self.every, resume=True, stream=self.stream)
        self.iterations += self.every
