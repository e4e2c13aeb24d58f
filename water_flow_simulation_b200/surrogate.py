"""Learned warm start: a 3D convolutional encoder-decoder that predicts a boat case's mean flow.

No counterpart in the reference, which starts every run from its 1D inlet profile
(floodsim/lbm3d.py:362-364).  The network works on a coarse copy of the lattice (blocks of
4x4x4 cells) and predicts, per coarse voxel, the departure of the time-averaged flow from
that 1D start: (ux - u_inlet(y, z), uy, uz, rho - 1).  `lift` turns the prediction into the
equilibrium populations and fields of a new start state (LBM3D.load_populations), from which
the unmodified LBM runs on.

Network (about 1.0M parameters, bf16 weights, float32 accumulation; every convolution,
forward and backward, is a GEMM on the tensor cores, lbm_gemm_bf16):
    a1 = relu(conv3 8->64 x)                      full coarse grid
    p  = pool2(a1)                                half grid
    a4 = relu(conv3 128->64 relu(conv3 128->128 relu(conv3 64->128 p)))
    u  = up2(a4) + a1                              full grid, skip connection
    out = conv3 64->8 relu(conv3 64->64 u)        channels 0..3 used
Trained with Adam on masked mean-square error against LBM steady states (time averages).
The CPU oracle of the same network is oracle/surrogate_oracle.py (used by the tests only).
"""
from __future__ import annotations

import math

import numpy as np

from . import _native as nat

LAYERS = (("c1", 8, 64, True), ("c2", 64, 128, True), ("c3", 128, 128, True), ("c4", 128, 64, True),
          ("c5", 64, 64, True), ("c6", 64, 8, False))
N_IN, N_OUT, N_PRED = 8, 8, 4
FACTOR = 4                      # fine cells per coarse voxel along each axis
# feature and target scales (lattice units -> O(1))
U_SCALE = 0.1
RHO_SCALE = 0.01
FORCE_SCALE = 1.0e3
CF_SCALE = 100.0


def _r8(n):
    return (n + 7) // 8 * 8


def coarse_dims(nz, ny, nx):
    """(Z, Y, X) of the coarse grid: ceil(n / FACTOR), rounded up to even (one 2x pooling level)."""
    return tuple(((n + FACTOR - 1) // FACTOR + 1) // 2 * 2 for n in (nz, ny, nx))


def _block_mean(a, dims, weight=None):
    """Mean over FACTOR^3 blocks of a (C, nz, ny, nx) array, zero-padded to the coarse grid
    (weighted by `weight` (nz, ny, nx) when given); returns (C, Z, Y, X)."""
    C = a.shape[0]
    Z, Y, X = dims
    pad = np.zeros((C, Z * FACTOR, Y * FACTOR, X * FACTOR))
    pad[:, :a.shape[1], :a.shape[2], :a.shape[3]] = a if weight is None else a * weight
    s = pad.reshape(C, Z, FACTOR, Y, FACTOR, X, FACTOR).sum(axis=(2, 4, 6))
    if weight is None:
        return s / FACTOR ** 3
    w = np.zeros((Z * FACTOR, Y * FACTOR, X * FACTOR))
    w[:weight.shape[0], :weight.shape[1], :weight.shape[2]] = weight
    n = w.reshape(Z, FACTOR, Y, FACTOR, X, FACTOR).sum(axis=(1, 3, 5))
    return s / np.maximum(n, 1.0)


def case_features(solid, Fx, Fy, Fz, uin_lb, cf=None):
    """Network input (V, 8) float32 and the coarse grid (Z, Y, X) of one case: fluid fraction,
    body force, 1D inlet speed, wall friction coefficient, x and z position."""
    nz, ny, nx = solid.shape
    dims = coarse_dims(nz, ny, nx)
    fl = (~np.asarray(solid, bool)).astype(np.float64)
    u1 = np.broadcast_to(np.asarray(uin_lb, np.float64).reshape(nz, ny, 1), (nz, ny, nx)) * fl
    cfa = np.zeros((nz, ny, nx)) if cf is None else np.asarray(cf, np.float64)
    x = np.broadcast_to(np.arange(nx) / max(nx - 1, 1), (nz, ny, nx))
    z = np.broadcast_to((np.arange(nz) / max(nz - 1, 1))[:, None, None], (nz, ny, nx))
    fine = np.stack([fl, np.asarray(Fx) * FORCE_SCALE * FACTOR ** 3, np.asarray(Fy) * FORCE_SCALE * FACTOR ** 3,
                     np.asarray(Fz) * FORCE_SCALE * FACTOR ** 3, u1 / U_SCALE, cfa * CF_SCALE, x * fl, z * fl])
    c = _block_mean(fine, dims)
    return np.ascontiguousarray(c.reshape(N_IN, -1).T, np.float32), dims


def case_targets(solid, uin_lb, rho, ux, uy, uz):
    """Training target (V, 4) float32 and mask (V,) from a case's mean fields (lattice units)."""
    nz, ny, nx = solid.shape
    dims = coarse_dims(nz, ny, nx)
    fl = (~np.asarray(solid, bool)).astype(np.float64)
    u1 = np.broadcast_to(np.asarray(uin_lb, np.float64).reshape(nz, ny, 1), (nz, ny, nx))
    sh = (nz, ny, nx)
    fine = np.stack([(np.asarray(ux).reshape(sh) - u1) / U_SCALE, np.asarray(uy).reshape(sh) / U_SCALE,
                     np.asarray(uz).reshape(sh) / U_SCALE, (np.asarray(rho).reshape(sh) - 1.0) / RHO_SCALE])
    t = _block_mean(fine, dims, weight=fl)
    frac = _block_mean(fl[None], dims)[0]
    return (np.ascontiguousarray(t.reshape(N_PRED, -1).T, np.float32),
            np.ascontiguousarray((frac >= 0.5).reshape(-1), np.float32))


class SurrogateNet:
    """The network's parameters (float32 masters, bf16 copies, Adam moments) and its passes."""

    def __init__(self, device=None, seed=0):
        torch = nat.require_cuda()
        self.torch = torch
        self.lib = nat.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        g = torch.Generator().manual_seed(seed)
        self.p = {}
        for name, cin, cout, relu in LAYERS:
            fan = 27 * cin
            W = torch.randn(cout, fan, generator=g) * math.sqrt((2.0 if relu else 0.5) / fan)
            d = self.device
            self.p[name] = dict(W=W.to(d), b=torch.zeros(cout, device=d), Wb=W.to(d, torch.bfloat16),
                                mW=torch.zeros(cout, fan, device=d), sW=torch.zeros(cout, fan, device=d),
                                mb=torch.zeros(cout, device=d), sb=torch.zeros(cout, device=d),
                                dW=torch.zeros(cout, fan, device=d), db=torch.zeros(cout, device=d))
        self.steps = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.cache = {}
        self.out_scale = np.ones(N_PRED, np.float32)     # prediction units: target / out_scale

    @property
    def n_params(self):
        return sum(v["W"].numel() + v["b"].numel() for v in self.p.values())

    def _st(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _gemm(self, A, lda, B, ldb, M, N, K, D, ldd, epi, bias=None):
        nat.check(self.lib.lbm_gemm_bf16(A.data_ptr(), lda, B.data_ptr(), ldb, M, N, K, D.data_ptr(), ldd, epi,
                                         None if bias is None else bias.data_ptr(), self.err.data_ptr(), self._st()),
                  "lbm_gemm_bf16")

    # ------------------------------------------------------------------ forward
    def _conv(self, name, x, dims, f32_out=False):
        torch = self.torch
        _, cin, cout, relu = next(l for l in LAYERS if l[0] == name)
        Z, Y, X = dims
        V = Z * Y * X
        col = torch.empty(V, 27 * cin, dtype=torch.bfloat16, device=self.device)
        nat.check(self.lib.lbm_nn_im2col(x.data_ptr(), cin, X, Y, Z, col.data_ptr(), self._st()), "lbm_nn_im2col")
        P = self.p[name]
        if f32_out:
            y = torch.empty(V, cout, dtype=torch.float32, device=self.device)
            self._gemm(col, 27 * cin, P["Wb"], 27 * cin, V, cout, 27 * cin, y, cout, 4, P["b"])
        else:
            y = torch.empty(V, cout, dtype=torch.bfloat16, device=self.device)
            self._gemm(col, 27 * cin, P["Wb"], 27 * cin, V, cout, 27 * cin, y, cout, 3 if relu else 2, P["b"])
        self.cache[name] = (col, y, dims, cin, cout, relu)
        return y

    def forward(self, x, dims):
        """x: (V, 8) float32 or bf16 on the device, V = Z*Y*X; returns (V, 8) float32."""
        torch = self.torch
        x = x.to(self.device, torch.bfloat16).contiguous()
        Z, Y, X = dims
        half = (Z // 2, Y // 2, X // 2)
        a1 = self._conv("c1", x, dims)
        p = torch.empty(half[0] * half[1] * half[2], 64, dtype=torch.bfloat16, device=self.device)
        nat.check(self.lib.lbm_nn_pool2(a1.data_ptr(), 64, X, Y, Z, p.data_ptr(), self._st()), "lbm_nn_pool2")
        a4 = self._conv("c4", self._conv("c3", self._conv("c2", p, half), half), half)
        u = torch.empty_like(a1)
        nat.check(self.lib.lbm_nn_up2_add(a4.data_ptr(), a1.data_ptr(), 64, X, Y, Z, u.data_ptr(), self._st()),
                  "lbm_nn_up2_add")
        return self._conv("c6", self._conv("c5", u, dims), dims, f32_out=True)

    # ------------------------------------------------------------------ backward
    def _conv_back(self, name, dy, need_dx=True):
        torch = self.torch
        col, y, dims, cin, cout, relu = self.cache[name]
        Z, Y, X = dims
        V = Z * Y * X
        Vp = _r8(V)
        P = self.p[name]
        st = self._st()
        g = torch.empty(V, cout, dtype=torch.bfloat16, device=self.device)
        nat.check(self.lib.lbm_nn_act_grad(dy.data_ptr(), y.data_ptr() if relu else None, V, cout, int(relu),
                                           g.data_ptr(), P["db"].data_ptr(), st), "lbm_nn_act_grad")
        gT = torch.empty(cout, Vp, dtype=torch.bfloat16, device=self.device)
        colT = torch.empty(27 * cin, Vp, dtype=torch.bfloat16, device=self.device)
        nat.check(self.lib.lbm_nn_transpose(g.data_ptr(), V, cout, Vp, gT.data_ptr(), st), "lbm_nn_transpose")
        nat.check(self.lib.lbm_nn_transpose(col.data_ptr(), V, 27 * cin, Vp, colT.data_ptr(), st), "lbm_nn_transpose")
        self._gemm(gT, Vp, colT, Vp, cout, 27 * cin, Vp, P["dW"], 27 * cin, 1)          # dW += g^T col
        if not need_dx:
            return None
        Wt = torch.empty(27 * cin, cout, dtype=torch.bfloat16, device=self.device)
        nat.check(self.lib.lbm_nn_transpose(P["Wb"].data_ptr(), cout, 27 * cin, cout, Wt.data_ptr(), st),
                  "lbm_nn_transpose")
        dcol = torch.empty(V, 27 * cin, dtype=torch.float32, device=self.device)
        self._gemm(g, cout, Wt, cout, V, 27 * cin, cout, dcol, 27 * cin, 0)             # dcol = g W
        dx = torch.empty(V, cin, dtype=torch.float32, device=self.device)
        nat.check(self.lib.lbm_nn_col2im(dcol.data_ptr(), cin, X, Y, Z, dx.data_ptr(), st), "lbm_nn_col2im")
        return dx

    def zero_grad(self):
        for P in self.p.values():
            P["dW"].zero_()
            P["db"].zero_()

    def loss_and_grad(self, x, dims, target, mask):
        """Forward, masked MSE against target (V, 4) and backward; gradients are added to dW/db."""
        torch = self.torch
        out = self.forward(x, dims)
        Z, Y, X = dims
        V = Z * Y * X
        target = target.to(self.device, torch.float32).contiguous()
        mask = mask.to(self.device, torch.float32).contiguous()
        n = max(float(mask.sum()), 1.0)
        dout = torch.empty_like(out)
        loss = torch.zeros(1, device=self.device)
        nat.check(self.lib.lbm_nn_mse(out.data_ptr(), N_OUT, target.data_ptr(), N_PRED, mask.data_ptr(), V, 1.0 / n,
                                      dout.data_ptr(), loss.data_ptr(), self._st()), "lbm_nn_mse")
        half = (Z // 2, Y // 2, X // 2)
        d5 = self._conv_back("c6", dout)
        du = self._conv_back("c5", d5)
        d4 = torch.empty(half[0] * half[1] * half[2], 64, dtype=torch.float32, device=self.device)
        nat.check(self.lib.lbm_nn_up2_back(du.data_ptr(), 64, X, Y, Z, d4.data_ptr(), self._st()), "lbm_nn_up2_back")
        dp = self._conv_back("c2", self._conv_back("c3", self._conv_back("c4", d4)))
        nat.check(self.lib.lbm_nn_pool2_back(dp.data_ptr(), 64, X, Y, Z, du.data_ptr(), 1, self._st()),
                  "lbm_nn_pool2_back")                                                 # da1 = du + pool'(dp)
        self._conv_back("c1", du, need_dx=False)
        self.cache = {}
        return loss, out

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.steps += 1
        st = self._st()
        for P in self.p.values():
            nat.check(self.lib.lbm_nn_adam(P["W"].data_ptr(), P["dW"].data_ptr(), P["mW"].data_ptr(), P["sW"].data_ptr(),
                                           P["W"].numel(), lr, b1, b2, eps, self.steps, P["Wb"].data_ptr(), st),
                      "lbm_nn_adam")
            nat.check(self.lib.lbm_nn_adam(P["b"].data_ptr(), P["db"].data_ptr(), P["mb"].data_ptr(), P["sb"].data_ptr(),
                                           P["b"].numel(), lr, b1, b2, eps, self.steps, None, st), "lbm_nn_adam")

    def check(self):
        """Raise if any tensor-core tile reported a timed-out wait."""
        if int(self.err.item()):
            raise nat.LBMError("a tensor-core GEMM tile timed out waiting for its operations")

    # ------------------------------------------------------------------ persistence
    def state(self):
        return {k: {"W": v["W"].cpu(), "b": v["b"].cpu()} for k, v in self.p.items()}

    @classmethod
    def load(cls, path=None, device=None):
        """A network with the weights saved by train_warmstart (default: the package's trained copy)."""
        import os
        path = path or os.path.join(os.path.dirname(__file__), "data", "warmstart_net.npz")
        z = np.load(path)
        net = cls(device=device)
        net.load_state({name: {"W": z[f"{name}_W"], "b": z[f"{name}_b"]} for name, _, _, _ in LAYERS})
        if "out_scale" in z:
            net.out_scale = z["out_scale"].astype(np.float32)
        return net

    def load_state(self, st):
        torch = self.torch
        for k, v in st.items():
            P = self.p[k]
            P["W"].copy_(torch.as_tensor(v["W"]))
            P["b"].copy_(torch.as_tensor(v["b"]))
            P["Wb"].copy_(P["W"].to(torch.bfloat16))


def gemm_throughput(M=32768, N=128, K=3456, reps=20, device=None):
    """TFLOP/s of lbm_gemm_bf16 on an M x N x K product (the forward GEMM of the 128 -> 128
    convolution on M coarse voxels), CUDA events around `reps` launches after a warm-up."""
    torch = nat.require_cuda()
    lib = nat.load()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(0)
    A = torch.randn(M, K, device=dev, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device=dev, generator=g).to(torch.bfloat16)
    D = torch.empty(M, N, dtype=torch.bfloat16, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream

    def run():
        nat.check(lib.lbm_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, D.data_ptr(), N, 3, None,
                                    err.data_ptr(), st), "lbm_gemm_bf16")
    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    if int(err.item()):
        raise nat.LBMError("a GEMM tile timed out")
    return dict(M=M, N=N, K=K, ms=ms, tflops=2.0 * M * N * K / (ms * 1e-3) / 1e12)
