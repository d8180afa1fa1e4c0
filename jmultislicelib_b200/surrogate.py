"""Learned control variate for frozen-phonon averaging.

A frozen-phonon STEM signal is the mean over phonon configurations c of the
multislice signal f(c) at each probe position.  A cheap surrogate g(c),
correlated with f(c), gives the unbiased estimate

    F_cv = mean_{c in all M} g(c) + mean_{c in n << M} (f(c) - g(c)),

whose variance is var(f - g) / n instead of var(f) / n for the plain mean of
n full multislice runs.  The surrogate here is a small convolutional network:
input a patch of the projected potential around the probe with one channel
per depth bin (the mean potential of the bin's slices in configuration c; the
workload uses one bin per readout interval, and the patch is a 64 x 64-pixel
window around the probe averaged to 16 x 16), output the integrated detector
signals at the readout thicknesses.  Depth-resolved inputs matter: for a weak
phase object the phonon fluctuation of a signal is close to a linear
functional of the potential fluctuation at each depth, with a depth-dependent
kernel, so depth-averaged inputs lose most of it.  Only g's fluctuation from configuration to
configuration matters, so it is trained on deviations: the patch minus its
mean over the configurations at that position, mapped to the signal minus
its mean.  It is trained on (patch, signal) pairs that the
multislice itself produces, with the library's own BF16 kernels
(csrc/jms_nn.cu); PyTorch only provides device memory.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

CONV = ((3, 16), (16, 32), (32, 64), (64, 64))   # (Ci, Co) of the four 3x3 / stride-2 convolutions
PATCH = 64


class SurrogateNet:
    """Conv(cin->16) -> Conv(16->32) -> Conv(32->64) -> Conv(64->64) (stride 2, ReLU unless relu=False) ->
    mean pool -> Linear(64->nout), on cin x size x size inputs.  On 16 x 16 inputs the last convolution
    leaves one pixel, so the linear layer reads position-specific features of the whole patch (a mean
    pool over a larger map would average the kernel over positions).  Without the ReLUs the network is a
    linear map of its input with a convolutional structure."""

    def __init__(self, nout: int, batch_max: int, seed: int = 0, cin: int = 3, size: int = PATCH, relu: bool = True):
        import torch

        from . import lib

        self.L = lib()
        self.nout = nout
        self.B = batch_max
        self.relu = 1 if relu else 0
        self.conv = ((cin, CONV[0][1]),) + tuple(CONV[1:])
        self.size = size
        dev = torch.device("cuda")
        rng = np.random.default_rng(seed)
        self.params = []          # FP32 masters
        self.bf = []              # BF16 copies of conv weights
        for (ci, co) in self.conv:
            w = rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), (co, ci, 3, 3)).astype(np.float32)
            self.params += [torch.from_numpy(w).to(dev), torch.zeros(co, dtype=torch.float32, device=dev)]
        c_last = self.conv[-1][1]
        wl = rng.normal(0.0, np.sqrt(1.0 / c_last), (nout, c_last)).astype(np.float32)
        self.params += [torch.from_numpy(wl).to(dev), torch.zeros(nout, dtype=torch.float32, device=dev)]
        self.bf = [self.params[2 * k].to(torch.bfloat16) for k in range(len(self.conv))]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.step = 0
        B = batch_max
        h = size
        self.act = []
        self.dact = []
        for (ci, co) in self.conv:
            h //= 2
            self.act.append(torch.zeros((B, co, h, h), dtype=torch.bfloat16, device=dev))
            self.dact.append(torch.zeros((B, co, h, h), dtype=torch.float32, device=dev))
        self.out = torch.zeros((B, nout), dtype=torch.float32, device=dev)
        self.dout = torch.zeros((B, nout), dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)

    def _stream(self):
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def forward(self, x, B: int):
        """x: BF16 [B, cin, size, size] on the device; returns out [B, nout] (a view)."""
        if not x.is_contiguous():
            raise ValueError("the surrogate reads its input as a C-ordered [B][C][H][W] array")
        L, s = self.L, self._stream()
        h = x
        size = self.size
        for k, (ci, co) in enumerate(self.conv):
            e = L.JMS_NnConvForward(h.data_ptr(), self.bf[k].data_ptr(), self.params[2 * k + 1].data_ptr(),
                                    self.act[k].data_ptr(), B, ci, size, size, co, self.relu, s)
            assert e == 0, e
            h = self.act[k]
            size //= 2
        c_last = self.conv[-1][1]
        e = L.JMS_NnPoolLinearForward(h.data_ptr(), self.params[-2].data_ptr(), self.params[-1].data_ptr(),
                                      self.out.data_ptr(), B, c_last, size * size, self.nout, s)
        assert e == 0, e
        return self.out[:B]

    def backward(self, x, t, B: int):
        """Gradients of the mean squared error of forward(x) against t into self.grads; returns the loss."""
        L, s = self.L, self._stream()
        out = self.forward(x, B)
        e = L.JMS_NnMseLoss(out.data_ptr(), t.data_ptr(), self.dout.data_ptr(), self.loss.data_ptr(),
                            B * self.nout, s)
        assert e == 0, e
        nl = len(self.conv)
        size = self.size >> nl
        c_last = self.conv[-1][1]
        e = L.JMS_NnPoolLinearBackward(self.act[-1].data_ptr(), self.params[-2].data_ptr(), self.dout.data_ptr(),
                                       self.dact[-1].data_ptr(), self.grads[-2].data_ptr(),
                                       self.grads[-1].data_ptr(), B, c_last, size * size, self.nout, s)
        assert e == 0, e
        for k in reversed(range(nl)):
            ci, co = self.conv[k]
            hin = x if k == 0 else self.act[k - 1]
            size_in = self.size >> k
            dx = None if k == 0 else self.dact[k - 1].data_ptr()
            e = L.JMS_NnConvBackward(hin.data_ptr(), self.bf[k].data_ptr(), self.act[k].data_ptr(),
                                     self.dact[k].data_ptr(), dx, self.grads[2 * k].data_ptr(),
                                     self.grads[2 * k + 1].data_ptr(), B, ci, size_in, size_in, co, self.relu, s)
            assert e == 0, e
        return self.loss

    def train_step(self, x, t, B: int, lr: float):
        loss = self.backward(x, t, B)
        self.step += 1
        s = self._stream()
        for k, p in enumerate(self.params):
            pb = self.bf[k // 2].data_ptr() if (k % 2 == 0 and k // 2 < len(self.conv)) else None
            e = self.L.JMS_NnAdam(p.data_ptr(), self.grads[k].data_ptr(), self.m[k].data_ptr(), self.v[k].data_ptr(),
                                  pb, p.numel(), lr, 0.9, 0.999, 1e-8, self.step, s)
            assert e == 0, e
        return loss

    def predict(self, x_all):
        """Forward over a BF16 [n, cin, size, size] tensor in batches; returns a host array [n, nout]."""
        import torch

        n = x_all.shape[0]
        x_all = x_all.contiguous()
        out = np.zeros((n, self.nout), np.float32)
        for i in range(0, n, self.B):
            b = min(self.B, n - i)
            out[i:i + b] = self.forward(x_all[i:i + b], b).cpu().numpy()
        torch.cuda.synchronize()
        return out


# ---------------------------------------------------------------------------
# inputs: potential patches of a phonon configuration
# ---------------------------------------------------------------------------
def channel_maps(sp, nobj: int, nslice_types: int, var: np.ndarray, nbins: int = 3) -> np.ndarray:
    """[nbins, ny, nx]: the mean projected potential of the slices in each of
    nbins equal parts of the specimen depth, in configuration var (variant
    index per object slice).  Needs the specimen's potentials
    (make_specimen(..., keep_potential=True))."""
    objslc = np.arange(nobj) % nslice_types
    out = []
    for part in np.array_split(np.arange(nobj), nbins):
        acc = np.zeros(sp.potential[0].shape[1:])
        keys, counts = np.unique(np.stack([objslc[part], np.asarray(var)[part]], 1), axis=0, return_counts=True)
        for (t, v), c in zip(keys, counts):
            acc += c * sp.potential[int(t)][int(v)]
        out.append(acc / len(part))
    return np.stack(out)


def patches(maps: np.ndarray, pos: np.ndarray, a: float, b: float, window: int = PATCH, pool: int = 1) -> np.ndarray:
    """[npos, C, window / pool, window / pool]: periodic window x window-pixel
    patches of maps [C, ny, nx] centred on the probe positions pos [npos, 2]
    (nm), averaged over pool x pool pixel blocks."""
    c, ny, nx = maps.shape
    px = np.rint(pos[:, 0] / a * nx).astype(np.int64)
    py = np.rint(pos[:, 1] / b * ny).astype(np.int64)
    off = np.arange(window) - window // 2
    ix = (px[:, None] + off[None, :]) % nx
    iy = (py[:, None] + off[None, :]) % ny
    p = maps[:, iy[:, :, None], ix[:, None, :]].transpose(1, 0, 2, 3)
    if pool > 1:
        m = window // pool
        p = p.reshape(p.shape[0], c, m, pool, m, pool).mean(axis=(3, 5))
    return np.ascontiguousarray(p)


class DevicePatches:
    """The inputs of channel_maps + patches computed on the device
    (JMS_NnPatches): the specimen's potentials [ntype][nvar][ny][nx] stay on
    the device, and each call returns the patches of a batch of
    configurations at the probe positions."""

    def __init__(self, sp, nobj: int, nslice_types: int, pos: np.ndarray, nbins: int, window: int = PATCH,
                 pool: int = 1):
        import torch

        from . import lib

        self.L = lib()
        pot = np.stack([np.asarray(sp.potential[t], np.float32) for t in range(nslice_types)])
        self.ntype, self.nvar, self.ny, self.nx = pot.shape
        self.pot = torch.from_numpy(np.ascontiguousarray(pot)).cuda()
        self.objslc = torch.from_numpy((np.arange(nobj) % nslice_types).astype(np.int32)).cuda()
        px = np.rint(pos[:, 0] / sp.a * self.nx).astype(np.int64) % self.nx
        py = np.rint(pos[:, 1] / sp.b * self.ny).astype(np.int64) % self.ny
        self.pix = torch.from_numpy(np.stack([px, py], 1).astype(np.int32)).cuda()
        self.nobj, self.npos, self.nbins, self.window, self.pool = nobj, len(pos), nbins, window, pool

    def __call__(self, var: np.ndarray):
        """var [nconf][nobj] -> device tensor [nconf][npos][nbins][m][m] (float32)."""
        import torch

        var = np.ascontiguousarray(np.atleast_2d(var), np.int32)
        d_var = torch.from_numpy(var).cuda()
        m = self.window // self.pool
        out = torch.empty((var.shape[0], self.npos, self.nbins, m, m), dtype=torch.float32, device="cuda")
        e = self.L.JMS_NnPatches(self.pot.data_ptr(), self.ntype, self.nvar, self.nx, self.ny, self.objslc.data_ptr(),
                                 self.nobj, d_var.data_ptr(), var.shape[0], self.pix.data_ptr(), self.npos,
                                 self.nbins, self.window, self.pool, out.data_ptr(),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if e:
            raise RuntimeError(f"JMS_NnPatches returned {e}")
        return out


def signals(J, d_pos, npos: int, var: np.ndarray, planes) -> np.ndarray:
    """Integrated detector signals [npos, len(planes) * ndet] of one phonon
    configuration var at the device positions d_pos (one multislice pass each)."""
    import torch

    nd, ndet = J.num_det_planes(), J.L.GetDetNum()
    d_out = torch.zeros((npos, nd, ndet), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()      # the library works on its own stream
    vs = np.ascontiguousarray(var, np.int32)
    e = J.L.JMS_ScanGPUDevice(npos, d_pos.data_ptr(), 0.0, 1, vs.ctypes.data_as(C.POINTER(C.c_int)),
                              d_out.data_ptr(), None, 0)
    if e:
        raise RuntimeError(f"JMS_ScanGPUDevice returned {e}")
    torch.cuda.synchronize()
    return d_out[:, list(planes), :].reshape(npos, -1).cpu().numpy()


# ---------------------------------------------------------------------------
# training and the control-variate estimate
# ---------------------------------------------------------------------------
class ControlVariate:
    """Surrogate, the normalisations of its inputs and outputs, and the
    regression coefficient beta of each output (cov(f, g) / var(g) on held-out
    pairs), so that the estimate below never has more variance than the plain
    mean in expectation: var(f - beta g) = (1 - rho^2) var(f) at the optimum."""

    def __init__(self, nout: int, batch: int = 256, seed: int = 0, cin: int = 3, size: int = PATCH,
                 relu: bool = True):
        self.net = SurrogateNet(nout, batch, seed, cin=cin, size=size, relu=relu)
        self.batch = batch
        self.xm = self.xs = None
        self.ym = self.ys = None
        self.beta = np.ones(nout)

    def _x(self, p):
        import torch

        # the kernels read [n][C][H][W] in C order: a strided array must be copied
        # into that layout first (torch.from_numpy keeps numpy's strides)
        z = (p - self.xm[None, :, None, None]) / self.xs[None, :, None, None]
        return torch.from_numpy(np.ascontiguousarray(z, dtype=np.float32)).cuda().to(torch.bfloat16).contiguous()

    def fit(self, X: np.ndarray, Y: np.ndarray, Xval: np.ndarray, Yval: np.ndarray, epochs: int = 30,
            lr: float = 2e-3, seed: int = 0):
        """X [n, cin, size, size] patches, Y [n, nout] signals; the epoch with the lowest
        loss on (Xval, Yval) is kept, and beta is fitted there.  Returns
        (training loss, validation loss) per epoch."""
        import torch

        self.xm = X.mean(axis=(0, 2, 3))
        self.xs = X.std(axis=(0, 2, 3)) + 1e-30
        self.ym = Y.mean(axis=0)
        self.ys = Y.std(axis=0) + 1e-300
        xd = self._x(X)
        yd = torch.from_numpy(((Y - self.ym) / self.ys).astype(np.float32)).cuda()
        xv = self._x(Xval)
        zv = (Yval - self.ym) / self.ys
        rng = np.random.default_rng(seed)
        n = X.shape[0]
        hist, best, best_state = [], np.inf, None
        for ep in range(epochs):
            order = torch.from_numpy(rng.permutation(n)).cuda()
            tot, nb = 0.0, 0
            for i in range(0, n - self.batch + 1, self.batch):
                idx = order[i:i + self.batch]
                loss = self.net.train_step(xd[idx].contiguous(), yd[idx].contiguous(), self.batch, lr)
                tot += float(loss.item())
                nb += 1
            pv = self.net.predict(xv).astype(np.float64)
            vloss = float(((pv - zv) ** 2).mean())
            hist.append((tot / max(nb, 1), vloss))
            if vloss < best:
                best = vloss
                best_state = [p.clone() for p in self.net.params]
        for p, q in zip(self.net.params, best_state):
            p.copy_(q)
        for k in range(len(self.net.conv)):
            self.net.bf[k].copy_(self.net.params[2 * k].to(self.net.bf[k].dtype))
        g = self.predict(Xval)
        gc, fc = g - g.mean(axis=0), Yval - Yval.mean(axis=0)
        self.beta = (gc * fc).sum(axis=0) / np.maximum((gc * gc).sum(axis=0), 1e-300)
        return hist

    def predict(self, X: np.ndarray) -> np.ndarray:
        return self.net.predict(self._x(X)).astype(np.float64) * self.ys + self.ym


def cv_estimate(f_few: np.ndarray, g_few: np.ndarray, g_all: np.ndarray, beta=1.0) -> np.ndarray:
    """mean_few f - beta (mean_few g - mean_all g); arrays [nconfig, npos, nout],
    beta per output.  Unbiased for any beta fixed in advance."""
    return f_few.mean(axis=0) - beta * (g_few.mean(axis=0) - g_all.mean(axis=0))


def timed(fn):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = fn()
    torch.cuda.synchronize()
    return r, time.perf_counter() - t0
