"""Learned preconditioner: a 3-level U-Net on the node grid used as the
learned stage of flexible CG's preconditioner (pic_ife_solve with
PIC_SOLVER_FCG_UNET; the stages are described in include/picgpu.h).

Network (NHWC, BF16 activations and weights, FP32 accumulation):
    e0: 3x3 conv 8->32, 32->32             (H x W)
    e1: pool, 3x3 conv 32->64, 64->64      (H/2)
    b : pool, 3x3 conv 64->128, 128->128   (H/4)
    d1: up + concat e1, 3x3 conv 192->64, 64->64
    d0: up + concat e0, 3x3 conv 96->32, 32->32
    head: 1x1 conv 32->1 (FP32)
Inputs: residual t / s (s = RMS of t over unknown nodes), log eps_r, a
signed distance to the nearest object boundary, the Dirichlet mask.  Output:
N(t) = s * net(t / s) on unknown nodes, 0 on Dirichlet nodes.  The 3x3
convolutions run on the tensor cores (tcgen05, libpicunet.so), every other
network kernel is in libpicunet.so too; torch provides device memory, the
random fields of the synthetic pairs, and a handle on the library stream.

The network sees the residual left by the classical stages (smoothing and
coarse correction), t = r - A z2, and is trained to return the error that
remains, e - z2.  Training is online: after each warm-up step the solve's
pairs -- the residual of the warm start with the error the solve removed,
and (b, phi) -- pass through the classical stages into a ring buffer, and a
few Adam steps are taken on random crops of buffered pairs and of fresh
operator-consistent pairs (t = A e for random fields e).  The loss is
sum (z - e/s_e)^2 with s_e the RMS of the crop's target: flexible CG is
invariant to the scale of each preconditioned vector, so the network learns
the shape of the error only.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import api

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpicunet.so")

UNET_FPROP_RELU, UNET_DGRAD = 0, 1
UNET_RMS_BLOCKS = 592
UNET_RMS_SCRATCH = 2 * UNET_RMS_BLOCKS + 1

LAYERS = [("e0a", 8, 32), ("e0b", 32, 32), ("e1a", 32, 64), ("e1b", 64, 64), ("ba", 64, 128),
          ("bb", 128, 128), ("d1a", 192, 64), ("d1b", 64, 64), ("d0a", 96, 32), ("d0b", 32, 32)]
LEVEL = {"e0": 0, "e1": 1, "b": 2, "d1": 1, "d0": 0}

EXPORTS = ["unet_conv", "unet_wgrad", "unet_rms", "unet_features", "unet_pool", "unet_pool_bwd", "unet_upcat",
           "unet_upcat_bwd", "unet_relu_bwd", "unet_head", "unet_head_bwd", "unet_loss", "unet_output",
           "unet_adam", "unet_fill_f32", "unet_f32_to_bf16"]

_lib = None


def load() -> C.CDLL:
    """Load libpicunet.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libpicunet.so not built at {LIB_PATH}: run pic_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    v, i32, i64, d, f, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_float, C.c_size_t
    lib.unet_conv.argtypes = [i32, i32, i32, i32, i32, i32, v, v, v, v, v, sz, C.POINTER(sz), v]
    lib.unet_wgrad.argtypes = [i32, i32, i32, i32, i32, v, v, v, v]
    lib.unet_rms.argtypes = [i64, v, v, v, v, v]
    lib.unet_features.argtypes = [i32, i32, v, v, v, v, v]
    lib.unet_pool.argtypes = [i32, i32, i32, i32, v, v, v]
    lib.unet_pool_bwd.argtypes = [i32, i32, i32, i32, v, v, i32, v]
    lib.unet_upcat.argtypes = [i32, i32, i32, i32, i32, v, v, v, v]
    lib.unet_upcat_bwd.argtypes = [i32, i32, i32, i32, i32, v, v, v, i32, v]
    lib.unet_relu_bwd.argtypes = [i64, i32, v, v, v, v]
    lib.unet_head.argtypes = [i64, i32, v, v, v, v, v]
    lib.unet_head_bwd.argtypes = [i64, i32, v, v, v, v, v, v, v]
    lib.unet_loss.argtypes = [i64, v, v, v, v, v, v, v]
    lib.unet_output.argtypes = [i64, v, v, v, v, v]
    lib.unet_adam.argtypes = [i64, v, v, v, v, v, f, f, f, f, i32, v]
    lib.unet_fill_f32.argtypes = [i64, v, f, v]
    lib.unet_f32_to_bf16.argtypes = [i64, v, v, v]
    _lib = lib
    return lib


def _ck(rc, what):
    if rc != 0:
        raise RuntimeError(f"libpicunet {what} failed ({rc})")


def _p(t):
    return C.c_void_p(t.data_ptr())


class DeviceArray:
    """Zero-copy view of a raw device pointer for torch.as_tensor."""

    def __init__(self, ptr: int, n: int, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class UNet:
    """Parameters (FP32 masters + BF16 copies), activations, forward,
    backward and Adam, all through libpicunet.so."""

    def __init__(self, seed: int = 0, stream=None):
        import torch
        self.torch = torch
        self.lib = load()
        self.stream = stream
        g = torch.Generator().manual_seed(seed)
        self.params = {}
        for name, cin, cout in LAYERS:
            w = torch.randn(cout, 3, 3, cin, generator=g) * math.sqrt(2.0 / (9 * cin))
            self._add(name + ".w", w)
            self._add(name + ".b", torch.zeros(cout))
        self._add("head.w", torch.randn(32, generator=g) * math.sqrt(1.0 / 32))
        self._add("head.b", torch.zeros(1))
        self.t = 0
        self.shape = None
        self.ws = None

    def _add(self, name, t32):
        torch = self.torch
        p = t32.to("cuda", torch.float32).contiguous()
        self.params[name] = {"p": p, "bf": p.to(torch.bfloat16).contiguous(), "g": torch.zeros_like(p),
                             "m": torch.zeros_like(p), "v": torch.zeros_like(p)}

    def state(self) -> dict:
        return {k: v["p"].detach().cpu().clone() for k, v in self.params.items()}

    def load_state(self, state: dict):
        for k, v in state.items():
            self.params[k]["p"].copy_(v.to("cuda"))
            self.params[k]["bf"].copy_(self.params[k]["p"].to(self.torch.bfloat16))

    def _ensure(self, n, h, w):
        """Allocate activations (and their gradients) for an n x h x w batch."""
        if self.shape == (n, h, w):
            return
        torch = self.torch
        h1, w1 = (h + 1) // 2, (w + 1) // 2
        h2, w2 = (h1 + 1) // 2, (w1 + 1) // 2
        sh = {"x0": (n, h, w, 8), "e0a": (n, h, w, 32), "e0b": (n, h, w, 32), "p1": (n, h1, w1, 32),
              "e1a": (n, h1, w1, 64), "e1b": (n, h1, w1, 64), "p2": (n, h2, w2, 64),
              "ba": (n, h2, w2, 128), "bb": (n, h2, w2, 128), "u1": (n, h1, w1, 192),
              "d1a": (n, h1, w1, 64), "d1b": (n, h1, w1, 64), "u0": (n, h, w, 96),
              "d0a": (n, h, w, 32), "d0b": (n, h, w, 32)}
        self.a = {k: torch.zeros(s, dtype=torch.bfloat16, device="cuda") for k, s in sh.items()}
        self.ga = {k: torch.zeros(s, dtype=torch.bfloat16, device="cuda") for k, s in sh.items()}
        self.z = torch.zeros(n * h * w, dtype=torch.float32, device="cuda")
        self.gz = torch.zeros_like(self.z)
        self.dims = {0: (h, w), 1: (h1, w1), 2: (h2, w2)}
        self.shape = (n, h, w)
        need = 0
        for name, cin, cout in LAYERS:
            hh, ww = self.dims[LEVEL[name[:-1]]]
            for op in (UNET_FPROP_RELU, UNET_DGRAD):
                s = C.c_size_t(0)
                _ck(self.lib.unet_conv(op, n, hh, ww, cin, cout, None, None, None, None, None, 0, C.byref(s), None),
                    f"workspace query {name}")
                need = max(need, s.value)
        self.ws = torch.zeros(max(need, 256), dtype=torch.uint8, device="cuda")

    def _dims_of(self, name):
        w = self.params[name + ".w"]["p"]
        return w.shape[3], w.shape[0]

    def _conv(self, name, src, dst, level):
        n = self.shape[0]
        h, w = self.dims[level]
        cin, cout = self._dims_of(name)
        _ck(self.lib.unet_conv(UNET_FPROP_RELU, n, h, w, cin, cout, _p(self.a[src]),
                               _p(self.params[name + ".w"]["bf"]), _p(self.a[dst]),
                               _p(self.params[name + ".b"]["bf"]), _p(self.ws), self.ws.numel(), None,
                               self.stream), "fprop " + name)

    def forward(self):
        """x0 (filled by the caller) -> self.z (FP32, one value per pixel)."""
        L, st = self.lib, self.stream
        n, h, w = self.shape
        h1, w1 = self.dims[1]
        self._conv("e0a", "x0", "e0a", 0)
        self._conv("e0b", "e0a", "e0b", 0)
        _ck(L.unet_pool(n, h, w, 32, _p(self.a["e0b"]), _p(self.a["p1"]), st), "pool1")
        self._conv("e1a", "p1", "e1a", 1)
        self._conv("e1b", "e1a", "e1b", 1)
        _ck(L.unet_pool(n, h1, w1, 64, _p(self.a["e1b"]), _p(self.a["p2"]), st), "pool2")
        self._conv("ba", "p2", "ba", 2)
        self._conv("bb", "ba", "bb", 2)
        _ck(L.unet_upcat(n, h1, w1, 128, 64, _p(self.a["bb"]), _p(self.a["e1b"]), _p(self.a["u1"]), st), "up1")
        self._conv("d1a", "u1", "d1a", 1)
        self._conv("d1b", "d1a", "d1b", 1)
        _ck(L.unet_upcat(n, h, w, 64, 32, _p(self.a["d1b"]), _p(self.a["e0b"]), _p(self.a["u0"]), st), "up0")
        self._conv("d0a", "u0", "d0a", 0)
        self._conv("d0b", "d0a", "d0b", 0)
        _ck(L.unet_head(n * h * w, 32, _p(self.a["d0b"]), _p(self.params["head.w"]["p"]),
                        _p(self.params["head.b"]["p"]), _p(self.z), st), "head")
        return self.z

    def _back_conv(self, name, inp, out, level, need_dx=True):
        """Gradient at `out` (post-ReLU) -> bias/weight gradients and the
        gradient at `inp`."""
        L, st = self.lib, self.stream
        n = self.shape[0]
        h, w = self.dims[level]
        P = self.params
        cin, cout = self._dims_of(name)
        _ck(L.unet_relu_bwd(n * h * w, cout, _p(self.a[out]), _p(self.ga[out]), _p(P[name + ".b"]["g"]), st),
            "relu_bwd " + name)
        _ck(L.unet_wgrad(n, h, w, cin, cout, _p(self.a[inp]), _p(self.ga[out]), _p(P[name + ".w"]["g"]), st),
            "wgrad " + name)
        if need_dx:
            _ck(L.unet_conv(UNET_DGRAD, n, h, w, cin, cout, _p(self.ga[out]), _p(P[name + ".w"]["bf"]),
                            _p(self.ga[inp]), None, _p(self.ws), self.ws.numel(), None, st), "dgrad " + name)

    def zero_grad(self):
        for v in self.params.values():
            _ck(self.lib.unet_fill_f32(v["g"].numel(), _p(v["g"]), 0.0, self.stream), "zero")

    def backward(self):
        """self.gz (dLoss/dz) -> parameter gradients (accumulated)."""
        L, st = self.lib, self.stream
        n, h, w = self.shape
        h1, w1 = self.dims[1]
        P = self.params
        _ck(L.unet_head_bwd(n * h * w, 32, _p(self.a["d0b"]), _p(P["head.w"]["p"]), _p(self.gz),
                            _p(self.ga["d0b"]), _p(P["head.w"]["g"]), _p(P["head.b"]["g"]), st), "head_bwd")
        self._back_conv("d0b", "d0a", "d0b", 0)
        self._back_conv("d0a", "u0", "d0a", 0)
        _ck(L.unet_upcat_bwd(n, h, w, 64, 32, _p(self.ga["u0"]), _p(self.ga["d1b"]), _p(self.ga["e0b"]), 0, st),
            "up0_bwd")
        self._back_conv("d1b", "d1a", "d1b", 1)
        self._back_conv("d1a", "u1", "d1a", 1)
        _ck(L.unet_upcat_bwd(n, h1, w1, 128, 64, _p(self.ga["u1"]), _p(self.ga["bb"]), _p(self.ga["e1b"]), 0,
                             st), "up1_bwd")
        self._back_conv("bb", "ba", "bb", 2)
        self._back_conv("ba", "p2", "ba", 2)
        _ck(L.unet_pool_bwd(n, h1, w1, 64, _p(self.ga["p2"]), _p(self.ga["e1b"]), 1, st), "pool2_bwd")
        self._back_conv("e1b", "e1a", "e1b", 1)
        self._back_conv("e1a", "p1", "e1a", 1)
        _ck(L.unet_pool_bwd(n, h, w, 32, _p(self.ga["p1"]), _p(self.ga["e0b"]), 1, st), "pool1_bwd")
        self._back_conv("e0b", "e0a", "e0b", 0)
        self._back_conv("e0a", "x0", "e0a", 0, need_dx=False)

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        for v in self.params.values():
            _ck(self.lib.unet_adam(v["p"].numel(), _p(v["p"]), _p(v["g"]), _p(v["m"]), _p(v["v"]), _p(v["bf"]),
                                   lr, b1, b2, eps, self.t, self.stream), "adam")


def static_features(mesh) -> np.ndarray:
    """Per-node [log eps_r, signed distance to the nearest object boundary in
    cells (clipped to +-8, scaled to +-1), Dirichlet mask] (FP32, [H*W*3])."""
    d = mesh.desc
    nnx, nny = mesh.nnx, mesh.nny
    xs = d.xmin + mesh.hx * np.arange(nnx)
    ys = d.ymin + mesh.hy * np.arange(nny)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    eps = np.ones((nnx, nny))
    dist = np.full((nnx, nny), np.inf)
    h = max(mesh.hx, mesh.hy)
    for k in range(d.n_objects):
        o = d.objects[k]
        if o.shape == api.PIC_SHAPE_CIRCLE:
            sd = (np.hypot(X - o.cx, Y - o.cy) - o.a) / h
        elif o.shape == api.PIC_SHAPE_ELLIPSE:
            c, s = math.cos(o.angle), math.sin(o.angle)
            u = (X - o.cx) * c + (Y - o.cy) * s
            v = -(X - o.cx) * s + (Y - o.cy) * c
            sd = (np.sqrt((u / o.a) ** 2 + (v / o.b) ** 2) - 1.0) * min(o.a, o.b) / h
        else:  # box: (cx, cy) lower-left, (a, b) upper-right corner
            dx = np.maximum(np.maximum(o.cx - X, X - o.a), 0.0)
            dy = np.maximum(np.maximum(o.cy - Y, Y - o.b), 0.0)
            inside = (X > o.cx) & (X < o.a) & (Y > o.cy) & (Y < o.b)
            sd = np.where(inside, -np.minimum(np.minimum(X - o.cx, o.a - X), np.minimum(Y - o.cy, o.b - Y)),
                          np.hypot(dx, dy)) / h
        dist = np.where(np.abs(sd) < np.abs(dist), sd, dist)
        if not o.conductor:
            eps = np.where(sd < 0, o.eps, eps)
    dist = np.clip(np.nan_to_num(dist, posinf=8.0), -8.0, 8.0) / 8.0
    mask = (mesh.array("node_type").reshape(nnx, nny) <= 0).astype(np.float64)
    f = np.stack([np.log(eps), dist, mask], axis=-1).astype(np.float32)
    return np.ascontiguousarray(f.reshape(-1))


class LearnedPreconditioner:
    """Configures flexible CG's preconditioner stages on a Simulation, serves
    the learned stage, and trains it online on the simulation's own solves.

    The learned stage (features, forward pass, output) is captured once into
    a CUDA graph on the library stream and replayed on every call: one launch
    and no host synchronisation per preconditioner application.
    """

    def __init__(self, sim, seed: int = 0, crop: int = 128, batch: int = 4, buffer: int = 32,
                 lr: float = 1e-3, synthetic: float = 0.5, smoothing: bool = True, omega: float = 2.0 / 3.0,
                 coarse_cells: int = 64, window: int = 4, use_graph: bool = True, multigrid: bool = False,
                 max_coarse_nodes: int = 4500):
        import torch
        self.torch = torch
        self.sim = sim
        self.lib = load()
        self.plib = sim.lib
        st = C.c_void_p()
        api.check(self.plib.pic_cuda_stream(C.byref(st)), "pic_cuda_stream")
        self.stream_ptr = st.value
        self.tstream = torch.cuda.ExternalStream(self.stream_ptr)
        self.H, self.W = sim.mesh.nnx, sim.mesh.nny
        self.npix = self.H * self.W
        nt = sim.mesh.array("node_type")
        self.mask = torch.tensor((nt > 0).astype(np.int32), device="cuda")
        self.mask_f = self.mask.to(torch.float64)
        self.feat = torch.tensor(static_features(sim.mesh), device="cuda")
        self.scale = torch.zeros(2, dtype=torch.float64, device="cuda")
        self.rms_scratch = torch.zeros(UNET_RMS_SCRATCH, dtype=torch.float64, device="cuda")
        self.net_full = UNet(seed=seed, stream=self.stream_ptr)
        self.net_full._ensure(1, self.H, self.W)
        self.crop, self.batch, self.lr = min(crop, self.H, self.W), batch, lr
        self.net_train = UNet(seed=seed, stream=self.stream_ptr)
        self.net_train.params = self.net_full.params  # shared weights, separate activations
        self.tr_scale = torch.zeros(batch, 2, dtype=torch.float64, device="cuda")
        self.tr_scale_e = torch.zeros(batch, 2, dtype=torch.float64, device="cuda")
        self.tr_scratch = torch.zeros(batch, UNET_RMS_SCRATCH, dtype=torch.float64, device="cuda")
        self.tr_loss = torch.zeros(2, dtype=torch.float64, device="cuda")
        self.synthetic = synthetic
        self.tgen = torch.Generator(device="cuda")
        self.tgen.manual_seed(seed)
        self.buf_t, self.buf_e = [], []
        self.cap = buffer
        self.rng = np.random.default_rng(seed)
        self.x_prev = torch.zeros(self.npix, dtype=torch.float64, device="cuda")
        self.losses = []
        self.calls = 0
        self.error = None
        self.use_graph = use_graph
        self.graphs = {}
        b = C.c_void_p()
        phi = C.c_void_p()
        api.check(self.plib.pic_solver_vectors(C.byref(b), C.byref(phi)), "pic_solver_vectors")
        self.b_dev = torch.as_tensor(DeviceArray(b.value, self.npix), device="cuda")
        self.phi_dev = torch.as_tensor(DeviceArray(phi.value, self.npix), device="cuda")
        self.smoothing, self.omega = int(smoothing), omega
        api.check(self.plib.pic_set_precond_stages(self.smoothing, omega, 1), "pic_set_precond_stages")
        # the classical coarse stage the network learns to complement: the
        # two-level space, or the multigrid V-cycle
        if multigrid:
            api.check(self.plib.pic_multigrid_setup(sim.mesh.ptr, max_coarse_nodes), "pic_multigrid_setup")
        else:
            api.check(self.plib.pic_coarse_setup(sim.mesh.ptr, coarse_cells), "pic_coarse_setup")
        self.multigrid = multigrid
        api.check(self.plib.pic_set_fcg_window(window), "pic_set_fcg_window")
        self._cb = api.PRECOND_FN(self._apply)
        api.check(self.plib.pic_set_preconditioner(self._cb, None), "pic_set_preconditioner")
        torch.cuda.synchronize()  # tensors above were filled on torch's default stream

    # ---- the learned stage --------------------------------------------------
    def apply_eager(self, t_ptr: int, y_ptr: int):
        """y = N(t) for device pointers t, y ([H*W] FP64), on the library stream."""
        L, st, net = self.lib, self.stream_ptr, self.net_full
        _ck(L.unet_rms(self.npix, C.c_void_p(t_ptr), _p(self.mask), _p(self.rms_scratch), _p(self.scale), st),
            "rms")
        _ck(L.unet_features(self.H, self.W, C.c_void_p(t_ptr), _p(self.scale), _p(self.feat), _p(net.a["x0"]), st),
            "features")
        net.forward()
        _ck(L.unet_output(self.npix, _p(net.z), _p(self.scale), _p(self.mask), C.c_void_p(y_ptr), st), "output")

    def _apply(self, t_ptr, y_ptr, user):
        try:
            self.calls += 1
            key = (t_ptr, y_ptr)
            gph = self.graphs.get(key)
            if gph is not None:
                with self.torch.cuda.stream(self.tstream):
                    gph.replay()
                return 0
            self.apply_eager(t_ptr, y_ptr)
            if self.use_graph:
                torch = self.torch
                gph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(gph, stream=self.tstream, capture_error_mode="relaxed"):
                    self.apply_eager(t_ptr, y_ptr)
                self.graphs[key] = gph
            return 0
        except Exception as exc:  # reported to FCG as a failing stage (-> Jacobi-PCG)
            self.error = repr(exc)
            return 1

    def set_learned(self, on: bool):
        """Switch the learned stage on or off (the classical stages stay)."""
        api.check(self.plib.pic_set_precond_stages(self.smoothing, self.omega, int(on)), "stages")

    def enable(self):
        api.check(self.plib.pic_set_solver(api.PIC_SOLVER_FCG_UNET), "pic_set_solver")

    def disable(self):
        api.check(self.plib.pic_set_solver(api.PIC_SOLVER_JPCG), "pic_set_solver")

    # ---- training pairs -----------------------------------------------------
    def _op(self, v):
        out = self.torch.empty_like(v)
        api.check(self.plib.pic_apply_operator(_p(v), _p(out)), "pic_apply_operator")
        return out

    def to_learned_pair(self, r, e):
        """(r, e = A^-1 r) -> (t, e - z2) with z2 the classical stages' output
        and t = r - A z2: the learned stage's input and target."""
        z2 = self.torch.empty_like(r)
        api.check(self.plib.pic_precond_apply(0, _p(r), _p(z2)), "pic_precond_apply")
        return (r - self._op(z2)) * self.mask_f, (e - z2) * self.mask_f

    def synthetic_pair(self):
        """(r = A e, e) for a random field e of power-law spectrum |k|^-alpha,
        alpha ~ U[0, 4] (white noise to smooth), zero on Dirichlet nodes."""
        torch = self.torch
        H, W = self.H, self.W
        noise = torch.randn(H, W, dtype=torch.float64, device="cuda", generator=self.tgen)
        alpha = float(self.rng.uniform(0.0, 4.0))
        kx = torch.fft.fftfreq(H, dtype=torch.float64, device="cuda")
        ky = torch.fft.rfftfreq(W, dtype=torch.float64, device="cuda")
        k2 = kx[:, None] ** 2 + ky[None, :] ** 2 + (1.0 / max(H, W)) ** 2
        e = torch.fft.irfft2(torch.fft.rfft2(noise) * k2 ** (-alpha / 2), s=(H, W)).reshape(-1) * self.mask_f
        e = e / e.norm().clamp_min(1e-300)
        return self._op(e), e

    def before_step(self):
        with self.torch.cuda.stream(self.tstream):
            self.x_prev.copy_(self.phi_dev)

    def harvest(self):
        """Add the last solve's pairs, (b - A x_prev, phi - x_prev) and
        (b, phi), on unknown nodes, through the classical stages."""
        with self.torch.cuda.stream(self.tstream):
            xp = self.x_prev * self.mask_f
            ph = self.phi_dev * self.mask_f
            b = self.b_dev * self.mask_f
            self._push(*self.to_learned_pair((b - self._op(xp)) * self.mask_f, ph - xp))
            self._push(*self.to_learned_pair(b, ph))

    def after_step(self, train_iters: int = 4):
        """Harvest the step's pairs and take a few Adam steps."""
        self.harvest()
        for _ in range(train_iters):
            self.train_step()

    def _push(self, t, e):
        if len(self.buf_t) >= self.cap:
            k = int(self.rng.integers(len(self.buf_t)))
            self.buf_t[k].copy_(t)
            self.buf_e[k].copy_(e)
        else:
            self.buf_t.append(t.clone())
            self.buf_e.append(e.clone())

    def train_step(self) -> float | None:
        """One Adam step on `batch` random crops, each from a buffered pair or
        (with probability `synthetic`) a fresh synthetic one.  Returns
        sum (z - e/s_e)^2 / sum (e/s_e)^2 over the batch."""
        if not self.buf_t and self.synthetic <= 0.0:
            return None
        torch = self.torch
        net, L, st = self.net_train, self.lib, self.stream_ptr
        c, n = self.crop, self.batch
        with torch.cuda.stream(self.tstream):
            net._ensure(n, c, c)
            net.zero_grad()
            self.tr_loss.zero_()
            crops = []
            for k in range(n):
                if not self.buf_t or self.rng.uniform() < self.synthetic:
                    tf, ef = self.to_learned_pair(*self.synthetic_pair())
                else:
                    j = int(self.rng.integers(len(self.buf_t)))
                    tf, ef = self.buf_t[j], self.buf_e[j]
                i0 = int(self.rng.integers(0, self.H - c + 1))
                j0 = int(self.rng.integers(0, self.W - c + 1))
                t = tf.view(self.H, self.W)[i0:i0 + c, j0:j0 + c].contiguous()
                e = ef.view(self.H, self.W)[i0:i0 + c, j0:j0 + c].contiguous()
                m = self.mask.view(self.H, self.W)[i0:i0 + c, j0:j0 + c].contiguous()
                f = self.feat.view(self.H, self.W, 3)[i0:i0 + c, j0:j0 + c].contiguous()
                sc, se = self.tr_scale[k], self.tr_scale_e[k]
                _ck(L.unet_rms(c * c, _p(t), _p(m), _p(self.tr_scratch[k]), _p(sc), st), "rms")
                _ck(L.unet_rms(c * c, _p(e), _p(m), _p(self.tr_scratch[k]), _p(se), st), "rms")
                _ck(L.unet_features(c, c, _p(t), _p(sc), _p(f), _p(net.a["x0"][k]), st), "features")
                crops.append((e, m, se))
            net.forward()
            for k, (e, m, se) in enumerate(crops):
                zk = net.z[k * c * c:(k + 1) * c * c]
                gk = net.gz[k * c * c:(k + 1) * c * c]
                _ck(L.unet_loss(c * c, _p(zk), _p(e), _p(se), _p(m), _p(gk), _p(self.tr_loss), st), "loss")
            net.backward()
            net.adam(self.lr)
            tl = self.tr_loss.cpu()
        rel = float(tl[0] / max(float(tl[1]), 1e-300))
        self.losses.append(rel)
        return rel
