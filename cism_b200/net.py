"""Learned initial guess: a 2-D U-Net on the vertex grid, in BF16.

The network maps five vertex fields of a domain -- ice thickness, the two
surface-slope components, log basal friction and the ice mask -- to the
(u, v) velocity on every sigma level (2 x nz channels, padded to a multiple
of 8).  Its guess replaces the zero or shallow-ice start of the Picard loop;
the unchanged solver then drives the solve to the same tolerance, so the
plain method remains both the fallback and the measure of the network's error.

Architecture (four resolution levels, 32/64/96/128 channels, 3 x 3 convs,
GELU, 2 x 2 average pooling, nearest upsampling, skip concatenation, a 1 x 1
head).  Weights and activations are BF16 with FP32 accumulation; the FP32
master weights and Adam moments live beside the BF16 GEMM copies.  Every
contraction and pointwise step runs in this project's kernels
(``csrc/net_kernels.cu``, loaded from ``libbpnet.so``); torch supplies device
memory and the stream.  Borders are periodic for doubly periodic domains and
zero otherwise.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import List, Optional, Sequence

import numpy as np

from . import configs

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libbpnet.so")
CHANNELS = (32, 64, 96, 128)
N_IN = 6  # input channels of the marine-family network (input_features); 5-input networks load too
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with make -C cism_b200/csrc")
        L = C.CDLL(LIB_PATH)
        vp, i, ll, f = C.c_void_p, C.c_int, C.c_longlong, C.c_float
        sig = {
            "bpnet_gemm_tn": [vp, vp, vp, vp, i, i, i, i, i, i, i, vp],
            "bpnet_gemm_tn_mma": [vp, vp, vp, vp, i, i, i, i, i, i, i, vp],
            "bpnet_gemm_tn_mode": [i, vp, vp, vp, vp, i, i, i, i, i, i, i, vp],
            "bpnet_gemm_status": [vp],
            "bpnet_im2col": [vp, vp, i, i, i, i, i, i, vp],
            "bpnet_col2im": [vp, vp, i, i, i, i, i, i, vp],
            "bpnet_transpose": [vp, vp, i, i, vp],
            "bpnet_act": [vp, vp, ll, i, i, i, i, vp],
            "bpnet_act_grad": [vp, vp, vp, ll, i, i, i, i, vp],
            "bpnet_to_bf16": [vp, vp, ll, vp],
            "bpnet_colsum": [vp, vp, ll, i, vp],
            "bpnet_pool": [vp, vp, i, i, i, i, vp],
            "bpnet_pool_grad": [vp, vp, i, i, i, i, i, i, vp],
            "bpnet_up": [vp, vp, i, i, i, i, i, i, vp],
            "bpnet_up_grad": [vp, vp, i, i, i, i, i, i, vp],
            "bpnet_copy_slice": [vp, vp, ll, i, i, i, vp],
            "bpnet_add_slice": [vp, vp, ll, i, i, i, vp],
            "bpnet_mse": [vp, vp, vp, vp, vp, ll, i, f, vp],
            "bpnet_adam": [vp, vp, vp, vp, vp, ll, i, i, f, f, f, f, f, f, vp],
            "bpnet_unpad": [vp, vp, ll, i, i, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = L
    return _lib


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the learned guess runs on the GPU: no CUDA device")
    return torch


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _s():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


LAUNCHES = 0  # kernels launched through this module (every _ck follows one launch)


def _ck(rc, what):
    global LAUNCHES
    LAUNCHES += 1
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def ceil8(x: int) -> int:
    return (x + 7) // 8 * 8


GEMM_KERNELS = {"tma": 0, "tc": 1, "mma": 2}


def gemm_tn(A, B, out, bias, M, N, K, lda, ldb, ldc, accum=False, kernel=None):
    """out[M][N] (FP32) = A[M][K] . B[N][K]^T (+ bias) (+ out); BF16 operands.
    kernel None: the library's default (tcgen05, TMA-fed); "tma", "tc" (tcgen05
    with register-staged operands) or "mma" (mma.sync) to choose."""
    if kernel is None:
        rc = lib().bpnet_gemm_tn(_p(A), _p(B), _p(out), _p(bias), M, N, K, lda, ldb, ldc, int(accum), _s())
    else:
        rc = lib().bpnet_gemm_tn_mode(GEMM_KERNELS[kernel], _p(A), _p(B), _p(out), _p(bias), M, N, K, lda, ldb,
                                      ldc, int(accum), _s())
    _ck(rc, "bpnet_gemm_tn")


def gemm_status() -> int:
    """1 if a bounded wait of the tcgen05 GEMM ran out since the last call."""
    return int(lib().bpnet_gemm_status(_s()))


def transpose(x, ldo: Optional[int] = None):
    """[R][Cc] BF16 -> [Cc][ldo] (columns past R zero)."""
    torch = _torch()
    R, Cc = x.shape
    ldo = ldo or R
    out = torch.zeros((Cc, ldo), dtype=torch.bfloat16, device=x.device)
    if ldo == R:
        _ck(lib().bpnet_transpose(_p(x), _p(out), R, Cc, _s()), "bpnet_transpose")
    else:
        tmp = torch.empty((Cc, R), dtype=torch.bfloat16, device=x.device)
        _ck(lib().bpnet_transpose(_p(x), _p(tmp), R, Cc, _s()), "bpnet_transpose")
        out[:, :R].copy_(tmp)
    return out


class Conv:
    """3 x 3 (or 1 x 1) convolution + bias + optional GELU."""

    def __init__(self, cin: int, cout: int, k3: bool, act: bool, rng: np.random.Generator):
        torch = _torch()
        assert cout % 8 == 0 and (k3 or cin % 8 == 0)
        self.cin, self.cout, self.k3, self.act = cin, cout, k3, act
        self.K = 9 * cin if k3 else cin
        self.Kp = ceil8(self.K)
        std = math.sqrt((2.0 if act else 0.25) / self.K)
        dev = "cuda"
        self.w = torch.tensor(rng.standard_normal((cout, self.K)) * std, dtype=torch.float32, device=dev)
        self.b = torch.zeros(cout, dtype=torch.float32, device=dev)
        self.wb = torch.zeros((cout, self.Kp), dtype=torch.bfloat16, device=dev)
        self.refresh()
        self.state = [torch.zeros_like(self.w), torch.zeros_like(self.w), torch.zeros_like(self.b),
                      torch.zeros_like(self.b)]
        self.gw = self.gb = None
        self.saved = None

    def refresh(self):
        self.wb.zero_()
        self.wb[:, :self.K].copy_(self.w.to(_torch().bfloat16))

    def params(self) -> int:
        return self.w.numel() + self.b.numel()

    def forward(self, x, shape, periodic: int, train: bool):
        """x: BF16 [P][cin]; returns (BF16 [P][cout], FP32 pre-activation)."""
        torch = _torch()
        B, H, W = shape
        P = B * H * W
        if self.k3:
            col = torch.empty((P, self.Kp), dtype=torch.bfloat16, device=x.device)
            _ck(lib().bpnet_im2col(_p(x), _p(col), B, H, W, self.cin, self.Kp, periodic, _s()), "im2col")
        else:
            col = x
        z = torch.empty((P, self.cout), dtype=torch.float32, device=x.device)
        gemm_tn(col, self.wb, z, self.b, P, self.cout, self.Kp, self.Kp, self.Kp, self.cout)
        y = torch.empty((P, self.cout), dtype=torch.bfloat16, device=x.device)
        _ck(lib().bpnet_act(_p(z), _p(y), P, self.cout, self.cout, 0, int(self.act), _s()), "act")
        self.saved = (col, z, shape, periodic) if train else None
        return y, z

    def backward(self, dy, need_dx: bool):
        """dy: FP32 [P][cout]; sets gw, gb; returns FP32 [P][cin] or None."""
        torch = _torch()
        col, z, (B, H, W), periodic = self.saved
        P = B * H * W
        dz = torch.empty((P, self.cout), dtype=torch.float32, device=dy.device)
        _ck(lib().bpnet_act_grad(_p(z), _p(dy), _p(dz), P, self.cout, self.cout, 0, int(self.act), _s()),
            "act_grad")
        self.gb = torch.empty(self.cout, dtype=torch.float32, device=dy.device)
        _ck(lib().bpnet_colsum(_p(dz), _p(self.gb), P, self.cout, _s()), "colsum")
        dzb = torch.empty((P, self.cout), dtype=torch.bfloat16, device=dy.device)
        _ck(lib().bpnet_to_bf16(_p(dz), _p(dzb), P * self.cout, _s()), "to_bf16")
        P8 = ceil8(P)
        dzt = transpose(dzb, P8)
        colt = transpose(col, P8)
        gwp = torch.empty((self.cout, self.Kp), dtype=torch.float32, device=dy.device)
        gemm_tn(dzt, colt, gwp, None, self.cout, self.Kp, P8, P8, P8, self.Kp)
        self.gw = torch.empty((self.cout, self.K), dtype=torch.float32, device=dy.device)
        _ck(lib().bpnet_unpad(_p(gwp), _p(self.gw), self.cout, self.K, self.Kp, _s()), "unpad")
        self.saved = None
        if not need_dx:
            return None
        wt = transpose(self.wb)  # [Kp][cout]
        dcol = torch.empty((P, self.Kp), dtype=torch.float32, device=dy.device)
        gemm_tn(dzb, wt, dcol, None, P, self.Kp, self.cout, self.cout, self.cout, self.Kp)
        if not self.k3:
            return dcol
        dx = torch.empty((P, self.cin), dtype=torch.float32, device=dy.device)
        _ck(lib().bpnet_col2im(_p(dcol), _p(dx), B, H, W, self.cin, self.Kp, periodic, _s()), "col2im")
        return dx

    def adam(self, lr: float, t: int, b1=0.9, b2=0.999, eps=1e-8):
        c1 = 1.0 / (1.0 - b1 ** t)
        c2 = 1.0 / (1.0 - b2 ** t)
        m1, m2, mb1, mb2 = self.state
        _ck(lib().bpnet_adam(_p(self.w), _p(self.gw), _p(m1), _p(m2), _p(self.wb), self.w.numel(), self.K,
                             self.Kp, lr, b1, b2, eps, c1, c2, _s()), "adam")
        _ck(lib().bpnet_adam(_p(self.b), _p(self.gb), _p(mb1), _p(mb2), None, self.b.numel(), 1, 1, lr, b1, b2,
                             eps, c1, c2, _s()), "adam")


class UNet:
    """The U-Net; ``n_out`` output channels (a multiple of 8)."""

    def __init__(self, n_out: int = 24, seed: int = 0, channels: Sequence[int] = CHANNELS, n_in: int = N_IN):
        rng = np.random.default_rng(seed)
        c = list(channels)
        self.channels = c
        self.n_out = n_out
        self.n_in = n_in
        self.enc = []
        cin = n_in
        for ch in c:
            self.enc.append([Conv(cin, ch, True, True, rng), Conv(ch, ch, True, True, rng)])
            cin = ch
        self.dec = []
        for lv in range(len(c) - 2, -1, -1):
            self.dec.append([Conv(c[lv + 1] + c[lv], c[lv], True, True, rng), Conv(c[lv], c[lv], True, True, rng)])
        self.head = Conv(c[0], n_out, False, False, rng)
        self.in_shift = np.zeros(n_in, np.float32)
        self.in_scale = np.ones(n_in, np.float32)
        self.out_scale = 1.0

    def convs(self) -> List[Conv]:
        return [cv for lv in self.enc for cv in lv] + [cv for lv in self.dec for cv in lv] + [self.head]

    def params(self) -> int:
        return sum(cv.params() for cv in self.convs())

    def forward(self, x, periodic: int, train: bool = False):
        """x: BF16 [B][H][W][n_in] (H, W multiples of 8); FP32 [B][H][W][n_out]."""
        torch = _torch()
        B, H, W, _ = x.shape
        assert H % 8 == 0 and W % 8 == 0
        nl = len(self.channels)
        shapes = [(B, H >> lv, W >> lv) for lv in range(nl)]
        cur = x.reshape(-1, self.n_in)
        skips = []
        for lv in range(nl):
            if lv > 0:
                b_, h_, w_ = shapes[lv - 1]
                pooled = torch.empty((b_ * (h_ // 2) * (w_ // 2), self.channels[lv - 1]), dtype=torch.bfloat16,
                                     device=x.device)
                _ck(lib().bpnet_pool(_p(cur), _p(pooled), b_, h_, w_, self.channels[lv - 1], _s()), "pool")
                cur = pooled
            for cv in self.enc[lv]:
                cur, _ = cv.forward(cur, shapes[lv], periodic, train)
            skips.append(cur)
        for di, lv in enumerate(range(nl - 2, -1, -1)):
            b_, h_, w_ = shapes[lv]
            cu, cs = self.channels[lv + 1], self.channels[lv]
            cat = torch.empty((b_ * h_ * w_, cu + cs), dtype=torch.bfloat16, device=x.device)
            _ck(lib().bpnet_up(_p(cur), _p(cat), b_, h_ // 2, w_ // 2, cu, cu + cs, 0, _s()), "up")
            _ck(lib().bpnet_copy_slice(_p(skips[lv]), _p(cat), b_ * h_ * w_, cs, cu + cs, cu, _s()), "copy")
            cur = cat
            for cv in self.dec[di]:
                cur, _ = cv.forward(cur, shapes[lv], periodic, train)
        _, z = self.head.forward(cur, shapes[0], periodic, train)
        return z.reshape(B, H, W, self.n_out)

    def backward(self, dout):
        """dout: FP32 [B][H][W][n_out] after a training forward; fills the gradients."""
        torch = _torch()
        nl = len(self.channels)
        B, H, W, _ = dout.shape
        shapes = [(B, H >> lv, W >> lv) for lv in range(nl)]
        d = self.head.backward(dout.reshape(-1, self.n_out), True)
        dskip = [None] * nl
        for lv in range(nl - 1):  # decoders in reverse order of application
            convs = self.dec[nl - 2 - lv]
            d = convs[1].backward(d, True)
            d = convs[0].backward(d, True)  # [P_lv][cu + cs]
            b_, h_, w_ = shapes[lv]
            cu, cs = self.channels[lv + 1], self.channels[lv]
            P = b_ * h_ * w_
            ds = torch.zeros((P, cs), dtype=torch.float32, device=dout.device)
            _ck(lib().bpnet_add_slice(_p(d), _p(ds), P, cs, cu + cs, cu, _s()), "add_slice")
            dskip[lv] = ds
            dup = torch.empty((P // 4, cu), dtype=torch.float32, device=dout.device)
            _ck(lib().bpnet_up_grad(_p(d), _p(dup), b_, h_ // 2, w_ // 2, cu, cu + cs, 0, _s()), "up_grad")
            d = dup  # gradient at the coarser level's output
        for lv in range(nl - 1, -1, -1):
            if lv < nl - 1:
                d = dskip[lv]
            convs = self.enc[lv]
            d = convs[1].backward(d, True)
            d = convs[0].backward(d, lv > 0)
            if lv > 0:
                b_, h_, w_ = shapes[lv - 1]
                _ck(lib().bpnet_pool_grad(_p(d), _p(dskip[lv - 1]), b_, h_, w_, self.channels[lv - 1],
                                          self.channels[lv - 1], 0, _s()), "pool_grad")

    def adam(self, lr: float, t: int):
        for cv in self.convs():
            cv.adam(lr, t)

    # -- persistence ---------------------------------------------------
    def state_dict(self) -> dict:
        out = {"channels": np.array(self.channels), "n_out": np.array(self.n_out),
               "in_shift": self.in_shift, "in_scale": self.in_scale, "out_scale": np.array(self.out_scale)}
        for i, cv in enumerate(self.convs()):
            out[f"w{i}"] = cv.w.cpu().numpy()
            out[f"b{i}"] = cv.b.cpu().numpy()
        return out

    def save(self, path: str):
        """The weights as .npz, and beside them the same as .bin for the C ABI."""
        np.savez_compressed(path, **self.state_dict())
        if path.endswith(".npz"):
            self.save_bin(path[:-4] + ".bin")

    def save_bin(self, path: str):
        """The weights in the flat binary form the C-ABI guess reads
        (bp_guess_load): magic "BPUNET1" + NUL; int32 version 1, n_in, n_out,
        levels, the channels, the number of convolutions; float32 in_shift
        [n_in], in_scale [n_in], out_scale; per convolution (encoder levels,
        decoder levels, head) int32 cin, cout, k3, act, K and float32 w
        [cout][K], b [cout].  Little-endian."""
        convs = self.convs()
        hdr = [1, self.n_in, self.n_out, len(self.channels)] + list(self.channels) + [len(convs)]
        with open(path, "wb") as f:
            f.write(b"BPUNET1\0")
            f.write(np.asarray(hdr, dtype="<i4").tobytes())
            f.write(np.asarray(self.in_shift, dtype="<f4").tobytes())
            f.write(np.asarray(self.in_scale, dtype="<f4").tobytes())
            f.write(np.asarray([self.out_scale], dtype="<f4").tobytes())
            for cv in convs:
                f.write(np.asarray([cv.cin, cv.cout, int(cv.k3), int(cv.act), cv.K], dtype="<i4").tobytes())
                f.write(np.ascontiguousarray(cv.w.cpu().numpy(), dtype="<f4").tobytes())
                f.write(np.ascontiguousarray(cv.b.cpu().numpy(), dtype="<f4").tobytes())

    @classmethod
    def load(cls, path: str) -> "UNet":
        torch = _torch()
        d = np.load(path)
        n_in = int(d["in_shift"].shape[0])
        net = cls(n_out=int(d["n_out"]), channels=tuple(int(c) for c in d["channels"]), n_in=n_in)
        for i, cv in enumerate(net.convs()):
            cv.w.copy_(torch.tensor(d[f"w{i}"]))
            cv.b.copy_(torch.tensor(d[f"b{i}"]))
            cv.refresh()
        net.in_shift = d["in_shift"].astype(np.float32)
        net.in_scale = d["in_scale"].astype(np.float32)
        net.out_scale = float(d["out_scale"])
        return net


def mse(y, t, mask):
    """Masked mean squared error of FP32 [B][H][W][C]; returns (loss, dL/dy)."""
    torch = _torch()
    P = y.shape[0] * y.shape[1] * y.shape[2]
    Cc = y.shape[3]
    count = float(mask.sum().item()) * Cc
    dy = torch.empty_like(y)
    part = torch.zeros(256, dtype=torch.float32, device=y.device)
    _ck(lib().bpnet_mse(_p(y), _p(t), _p(mask), _p(dy), _p(part), P, Cc, 1.0 / max(count, 1.0), _s()), "mse")
    return float(part.double().sum().item()), dy


# ---------------------------------------------------------------------
# fields of a domain on its owned vertex grid
# ---------------------------------------------------------------------
def _stag(a):
    return 0.25 * (a[:-1, :-1] + a[1:, :-1] + a[:-1, 1:] + a[1:, 1:])


def features(m: configs.BPModel) -> np.ndarray:
    """[ny_owned][nx_owned][5]: thickness (km), surface slope x and y
    (x 1000), log10 basal friction (Pa a/m, clamped to >= 1) and the ice mask
    at the owned vertices.  The surface enters through its gradient, which
    stays continuous across periodic seams where the surface itself jumps."""
    js, is_ = m.owned_vertex_slices()
    H = _stag(m.thck)
    s = m.usrf
    sx = (s[:-1, 1:] + s[1:, 1:] - s[:-1, :-1] - s[1:, :-1]) / (2.0 * m.dx)
    sy = (s[1:, :-1] + s[1:, 1:] - s[:-1, :-1] - s[:-1, 1:]) / (2.0 * m.dy)
    if m.beta_external is not None:
        beta = np.maximum(np.asarray(m.beta_external, np.float64), 1.0)
    else:
        beta = np.full(H.shape, 1.0e8)
    mask = (H > m.thklim).astype(np.float64)
    f = np.stack([H / 1000.0, sx * 1000.0, sy * 1000.0, np.log10(beta), mask], axis=-1)
    return f[js, is_]


def velocity_targets(m: configs.BPModel, u: np.ndarray, v: np.ndarray, n_out: int = 24) -> np.ndarray:
    """[ny_owned][nx_owned][n_out]: (u_k, v_k) per level, zero padded."""
    js, is_ = m.owned_vertex_slices()
    t = np.zeros(u[js, is_].shape[:2] + (n_out,))
    t[..., 0:2 * m.nz:2] = u[js, is_]
    t[..., 1:2 * m.nz:2] = v[js, is_]
    return t


def guess_from_output(m: configs.BPModel, out: np.ndarray):
    """Network output [ny_owned][nx_owned][>= 2 nz] -> halo'd (uvel, vvel)."""
    js, is_ = m.owned_vertex_slices()
    u = np.zeros(m.vshape3)
    v = np.zeros(m.vshape3)
    u[js, is_] = out[..., 0:2 * m.nz:2]
    v[js, is_] = out[..., 1:2 * m.nz:2]
    return configs.halo_fill_stag(u, m.periodic), configs.halo_fill_stag(v, m.periodic)


# ---------------------------------------------------------------------
# fields of a prepared solve (the outputs of bp_setup, which a caller of the
# C ABI also holds): the features of the marine-family network
# ---------------------------------------------------------------------
VOL0 = 1.0e9  # the solver's volume scale (glissade_velo_higher.F90:1111)


def input_features(m: configs.BPModel, arrays: dict, n_in: int = N_IN) -> np.ndarray:
    """[ny_owned][nx_owned][n_in] at the owned vertices from bp_setup's
    arrays: thickness stagthck (km), the driving stress -- the gravity load
    summed over the column, per horizontal area (1e5 Pa) -- in x and y,
    log10 of beta_internal (clamped to >= 1), the ice mask (+1 where
    beta_internal > 0, i.e. grounded ice, -1 floating ice, 0 no active
    vertex) and (sixth channel) log10 of the mean flow-law factor flwafact =
    0.5 A^(-1/n) over the layers of the vertex's active cells.  Zero at
    vertices that are not active.  The surface and bed enter through the
    driving stress and the grounded/floating mask: the load vector carries
    rho g H grad s and the calving-front pressure, and stays continuous across
    a periodic seam where the surface itself jumps.  The sums run in the
    device's order (level by level; cells SW, SE, NW, NE of the vertex, each
    layer by layer)."""
    js, is_ = m.owned_vertex_slices()
    act = np.asarray(arrays["active_vertex"])[js, is_] != 0
    H = np.asarray(arrays["stagthck"])[js, is_]
    lu = np.asarray(arrays["loadu"])[js, is_]
    lv = np.asarray(arrays["loadv"])[js, is_]
    su = np.zeros(H.shape)
    sv = np.zeros(H.shape)
    for k in range(lu.shape[-1]):
        su = su + lu[..., k]
        sv = sv + lv[..., k]
    area = VOL0 / (m.dx * m.dy) * 1.0e-5
    beta = np.asarray(arrays["beta_internal"])[js, is_]
    chans = [H / 1000.0, su * area, sv * area, np.log10(np.maximum(beta, 1.0)), np.where(beta > 0.0, 1.0, -1.0)]
    if n_in > 5:
        fl = np.asarray(arrays["flwafact"])
        ac = np.asarray(arrays["active_cell"]) != 0
        j0, j1, i0, i1 = js.start, js.stop, is_.start, is_.stop
        sf = np.zeros(H.shape)
        cnt = np.zeros(H.shape)
        for dj, di in ((0, 0), (0, 1), (1, 0), (1, 1)):  # the cells of which the vertex is the NE, NW, SE, SW corner
            a = ac[j0 + dj:j1 + dj, i0 + di:i1 + di]
            for k in range(fl.shape[-1]):
                sf = sf + np.where(a, fl[j0 + dj:j1 + dj, i0 + di:i1 + di, k], 0.0)
                cnt = cnt + np.where(a, 1.0, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            chans.append(np.where(cnt > 0, np.log10(np.where(cnt > 0, sf / np.maximum(cnt, 1.0), 1.0)), 0.0))
    f = np.stack(chans[:n_in], axis=-1)
    return np.where(act[..., None], f, 0.0)


def normalized_input(model: "UNet", f: np.ndarray) -> np.ndarray:
    """input_features (padded) -> the network's input: (f - in_shift) *
    in_scale at the active vertices (mask channel +-1), zero elsewhere."""
    act = (f[..., 4] != 0.0)[..., None]
    return np.where(act, (f - model.in_shift) * model.in_scale, 0.0)


def padded_shape(gy: int, gx: int):
    """The network's grid for an owned grid of gy x gx vertices: both sides
    rounded up to multiples of 8 (three 2 x 2 poolings)."""
    return ceil8(gy), ceil8(gx)


def pad_grid(f: np.ndarray) -> np.ndarray:
    """[gy][gx][C] -> [ceil8(gy)][ceil8(gx)][C], zero past the owned grid."""
    gy, gx = f.shape[:2]
    py, px = padded_shape(gy, gx)
    out = np.zeros((py, px) + f.shape[2:], dtype=f.dtype)
    out[:gy, :gx] = f
    return out


def guess_from_grid(m: configs.BPModel, out: np.ndarray, active: np.ndarray):
    """Network output on the padded grid [py][px][>= 2 nz] -> halo'd (uvel,
    vvel), zero at vertices that are not active."""
    js, is_ = m.owned_vertex_slices()
    u = np.zeros(m.vshape3)
    v = np.zeros(m.vshape3)
    gy, gx = u[js, is_].shape[:2]
    act = (np.asarray(active)[js, is_] != 0)[..., None]
    u[js, is_] = np.where(act, out[:gy, :gx, 0:2 * m.nz:2], 0.0)
    v[js, is_] = np.where(act, out[:gy, :gx, 1:2 * m.nz:2], 0.0)
    return configs.halo_fill_stag(u, m.periodic), configs.halo_fill_stag(v, m.periodic)


def predict(net: UNet, models: Sequence[configs.BPModel]):
    """Guesses (uvel, vvel) for domains of one owned-grid size and border type."""
    torch = _torch()
    feats = (np.stack([features(m) for m in models]) - net.in_shift) * net.in_scale
    periodic = int(models[0].periodic)
    x = torch.tensor(feats, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    out = net.forward(x, periodic, train=False).cpu().numpy() * net.out_scale
    return [guess_from_output(m, o) for m, o in zip(models, out)]


# ---------------------------------------------------------------------
# timing of the GEMM kernels on the U-Net's shapes
# ---------------------------------------------------------------------
GEMM_SHAPES = (("forward, level 0, input", 524288, 32, 56), ("forward, level 0", 524288, 32, 288),
               ("forward, level 1", 131072, 64, 576), ("forward, level 2", 32768, 96, 864),
               ("forward, level 3", 8192, 128, 1152), ("head", 524288, 24, 32),
               ("weight gradient, level 0", 32, 288, 524288), ("weight gradient, level 1", 64, 576, 131072),
               ("weight gradient, level 3", 128, 1152, 8192), ("input gradient, level 0", 524288, 288, 32),
               ("input gradient, level 1", 131072, 576, 64))


def gemm_timings(reps: int = 10):
    """CUDA-event time of every GEMM kernel on the products of one training
    step of the marine network (batch 8 of 256 x 256 grids), and its
    relative error against the FP32 product of the same BF16 operands."""
    torch = _torch()
    rows = []
    for name, M, N, K in GEMM_SHAPES:
        a = torch.randn(M, K, device="cuda").to(torch.bfloat16)
        b = torch.randn(N, K, device="cuda").to(torch.bfloat16)
        c = torch.empty(M, N, device="cuda")
        ref = a.float() @ b.float().T
        row = {"product": name, "M": M, "N": N, "K": K}
        for kern in GEMM_KERNELS:
            gemm_tn(a, b, c, None, M, N, K, K, K, N, kernel=kern)
            torch.cuda.synchronize()
            err = float((c - ref).norm() / ref.norm())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                gemm_tn(a, b, c, None, M, N, K, K, K, N, kernel=kern)
            e1.record()
            torch.cuda.synchronize()
            us = e0.elapsed_time(e1) / reps * 1e3
            row[kern] = {"us": round(us, 1), "tflops": round(2.0 * M * N * K / (us * 1e-6) / 1e12, 1),
                         "rel_err": float("%.2e" % err)}
        rows.append(row)
        del a, b, c, ref
    return rows


if __name__ == "__main__":
    import json
    import sys

    if sys.argv[1:] == ["gemm"]:
        for r in gemm_timings():
            print(json.dumps(r), flush=True)
        print(json.dumps({"gemm_status": gemm_status()}))
