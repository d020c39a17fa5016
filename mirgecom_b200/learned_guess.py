"""Learned initial guess for the mixture-temperature Newton solve.

An 8 -> 64 -> 64 -> 1 tanh network maps (internal energy, 7 mass fractions)
to a temperature.  Training and inference run on the device through the
library's own bf16 tensor-core kernels (``csrc/mlp.cu``): forward and
backward passes, split-K weight gradients and Adam.  The training pairs are
produced by the plain float64 Newton solve itself (``make_fluid_state`` with
a fixed, generous iteration count), on states drawn from the distributions
of the reacting benchmark: T ~ U[300, 2500] K, Y ~ Dirichlet(2).

The network only supplies the Newton starting point of the mixed-precision
form (``PyrometheusMixture(learned_guess=...)``); the plain guess (the
step-start temperature) remains the fallback whenever the float64 residual
check fails, so the converged temperatures meet the same tolerance with or
without the network.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from mirgecom_b200 import _lib

H = 64
KIN = 16
P_W1 = 0
P_B1 = P_W1 + H * KIN
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + H
NPARAM = P_B3 + 1


class TemperatureMLP:
    def __init__(self, device, seed=0, nspecies=7):
        if nspecies != 7:
            raise ValueError("the temperature network takes 7 mass fractions")
        lib = _lib.load()
        assert lib.mgc_mlp_nparams() == NPARAM
        self.device = device
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(NPARAM, dtype=torch.float32)
        w1 = torch.randn((H, 8), generator=g) * math.sqrt(1.0 / 8)
        p[P_W1:P_B1].view(H, KIN)[:, :8] = w1
        p[P_W2:P_B2] = (torch.randn((H, H), generator=g) * math.sqrt(1.0 / H)).ravel()
        p[P_W3:P_B3] = torch.randn(H, generator=g) * math.sqrt(1.0 / H)
        self.params = p.to(device)
        self.w1 = torch.zeros(H * KIN, dtype=torch.bfloat16, device=device)
        self.w2 = torch.zeros(H * H, dtype=torch.bfloat16, device=device)
        self.w2t = torch.zeros(H * H, dtype=torch.bfloat16, device=device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step_count = 0
        self.in_shift = np.zeros(8, dtype=np.float32)
        self.in_scale = np.ones(8, dtype=np.float32)
        self.out_shift = 1400.0
        self.out_scale = 1100.0
        with torch.cuda.device(device):
            _lib.check(lib.mgc_mlp_refresh(C.byref(self.struct()), _lib.stream_handle()),
                       "mgc_mlp_refresh")

    def struct(self) -> _lib.MLPStruct:
        s = _lib.MLPStruct()
        s.params = self.params.data_ptr()
        s.w1_bf16 = self.w1.data_ptr()
        s.w2_bf16 = self.w2.data_ptr()
        s.w2t_bf16 = self.w2t.data_ptr()
        for i in range(8):
            s.in_shift[i] = float(self.in_shift[i])
            s.in_scale[i] = float(self.in_scale[i])
        s.out_shift = float(self.out_shift)
        s.out_scale = float(self.out_scale)
        return s

    # {{{ data

    @staticmethod
    def training_pairs(mech, n, device, seed=0, t_range=(300.0, 2500.0), niter=30):
        """(e, Y, T) pairs: random states, temperature by the plain Newton."""
        from mirgecom_b200.eos import PyrometheusMixture
        from mirgecom_b200.fluid import ConservedVars
        from mirgecom_b200.gas_model import GasModel, make_fluid_state
        from mirgecom_b200.initializers import _nasa_e_rt
        from mirgecom_b200.thermochemistry import GAS_CONSTANT
        g = torch.Generator().manual_seed(seed)
        t = (t_range[0] + (t_range[1] - t_range[0]) * torch.rand(n, generator=g,
                                                                dtype=torch.float64))
        gam = -torch.log(torch.rand((mech.nspecies, 2, n), generator=g,
                                    dtype=torch.float64).clamp_min(1e-300)).sum(dim=1)
        y = gam / gam.sum(dim=0, keepdim=True)
        t, y = t.to(device), y.to(device)
        w = torch.as_tensor(mech.molecular_weights, dtype=torch.float64,
                            device=device)[:, None]
        e = GAS_CONSTANT * t * (y * _nasa_e_rt(mech, t) / w).sum(dim=0)
        rho = torch.ones_like(t)
        q = torch.cat([rho[None], (rho * e)[None], torch.zeros((3, n), dtype=torch.float64,
                                                               device=device), y])
        gas = GasModel(eos=PyrometheusMixture(mech, temperature_niter=niter))
        st = make_fluid_state(ConservedVars(q.contiguous(), 3), gas,
                              temperature_seed=torch.full_like(t, 1500.0))
        return e, y, st.temperature

    def set_normalisation(self, e, y):
        feats = torch.cat([e[None], y]).to(torch.float64)
        mu = feats.mean(dim=1).cpu().numpy()
        sd = feats.std(dim=1).clamp_min(1e-12).cpu().numpy()
        self.in_shift = mu.astype(np.float32)
        self.in_scale = (1.0 / sd).astype(np.float32)

    def features(self, e, y):
        f = torch.cat([e[None], y]).to(torch.float32)
        sh = torch.as_tensor(self.in_shift, device=f.device)[:, None]
        sc = torch.as_tensor(self.in_scale, device=f.device)[:, None]
        return ((f - sh) * sc).T.contiguous()          # [n][8]

    # }}}

    # {{{ training

    def loss_and_grad(self, x, t_norm):
        lib = _lib.load()
        n = x.shape[0]
        ws_bytes = lib.mgc_mlp_train_workspace_bytes(n)
        ws = getattr(self, "_ws", None)
        if ws is None or ws.numel() < ws_bytes:
            ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
            self._ws = ws
        with torch.cuda.device(self.device):
            _lib.check(lib.mgc_mlp_train_grad(
                n, _lib.ptr(x), _lib.ptr(t_norm), C.byref(self.struct()), _lib.ptr(ws),
                ws.numel(), _lib.ptr(self.grad), _lib.ptr(self.loss), _lib.stream_handle()),
                "mgc_mlp_train_grad")
        return self.loss, self.grad

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        lib = _lib.load()
        self.step_count += 1
        with torch.cuda.device(self.device):
            _lib.check(lib.mgc_mlp_adam(
                C.byref(self.struct()), _lib.ptr(self.grad), _lib.ptr(self.m),
                _lib.ptr(self.v), lr, beta1, beta2, eps, self.step_count,
                _lib.stream_handle()), "mgc_mlp_adam")

    def fit(self, e, y, t, steps=2000, batch=65536, lr=3e-3, seed=0):
        """Adam on mini-batches; returns the loss history (normalised MSE)."""
        self.set_normalisation(e, y)
        x_all = self.features(e, y)
        t_all = ((t.to(torch.float32) - self.out_shift) / self.out_scale).contiguous()
        n = x_all.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        hist = []
        for it in range(steps):
            idx = torch.randint(0, n, (min(batch, n),), generator=g, device=self.device)
            self.loss_and_grad(x_all[idx].contiguous(), t_all[idx].contiguous())
            frac = it / max(steps - 1, 1)
            self.adam_step(lr * 0.5 * (1 + math.cos(math.pi * frac)) + 1e-5)
            if it % 100 == 0 or it == steps - 1:
                hist.append(float(self.loss.item()))
        return hist

    # }}}

    def predict(self, cv):
        """Temperature guess for every node of a float32 ConservedVars."""
        lib = _lib.load()
        q = cv.q.contiguous()
        n = q[0].numel()
        out = torch.empty(q.shape[1:], dtype=torch.float32, device=q.device)
        with torch.cuda.device(q.device):
            _lib.check(lib.mgc_mlp_infer(cv.dim, cv.nspecies, n, _lib.ptr(q),
                                         C.byref(self.struct()), _lib.ptr(out),
                                         _lib.stream_handle()), "mgc_mlp_infer")
        return out

    def numpy_params(self):
        p = self.params.cpu().numpy().astype(np.float64)
        return {"w1": p[P_W1:P_B1].reshape(H, KIN)[:, :8], "b1": p[P_B1:P_W2],
                "w2": p[P_W2:P_B2].reshape(H, H), "b2": p[P_B2:P_W3],
                "w3": p[P_W3:P_B3], "b3": p[P_B3]}
