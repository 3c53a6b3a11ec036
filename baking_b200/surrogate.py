"""Learned surrogate of the Ding return map: MLP 7 -> 64 -> 64 -> 3 (SiLU), BF16 weights, FP32 accumulation.

Inputs per yielding particle: the three log singular values of the trial elastic gradient (sorted
descending), the effective temperature after the gelation latch, the water saturation, the gas
content and the plastic volume strain log(1 - n0 + n). Outputs: the return's change of the three
log principal strains (before the coupled-porosity volume correction), from which the returned
elastic gradient, the Kirchhoff stress and the end-state porosity follow exactly. The reference
has no learned component; its exact return map (physics/materials/ding.py:103-137,
porous_return.py:43-61) produces the training pairs, runs for particles outside the training
range, and judges the surrogate's error.

Training runs on the device through the library's own kernels: ``bk_mlp_gradient`` (forward +
backward, rounded like inference), ``bk_mlp_adam`` and ``bk_mlp_pack``; inference uses the tensor
cores (``bk_mlp_infer`` stand-alone, or fused into the substep's G2P kernel).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

P = C.c_void_p
FEATURES, OUTPUTS, PARAMS, PACKED_BYTES = 7, 3, 4867, 12864
FEATURE_NAMES = ("log_s1", "log_s2", "log_s3", "temperature", "saturation", "gas", "plastic_volume_strain")


class BkMlpNorm(C.Structure):
    _fields_ = [("in_mean", C.c_float * 8), ("in_scale", C.c_float * 8), ("out_scale", C.c_float * 4)]


SIGNATURES = {
    "bk_mlp_infer": [C.c_int64, P, P, P, P, P, P],
    "bk_mlp_gradient": [C.c_int64, P, P, P, P, P, P, P],
    "bk_mlp_adam": [P, P, P, P, C.c_int32, C.c_float, C.c_float, C.c_float, C.c_float, P],
    "bk_mlp_pack": [P, P, P],
}


def _lib_handle():
    lib = _lib.load()
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        if fn.argtypes != argtypes:
            fn.restype = C.c_int
            fn.argtypes = argtypes
    return lib


def _call(lib, name, *args):
    rc = getattr(lib, name)(*args)
    if rc != 0:
        raise RuntimeError(f"{name} failed ({rc}): {lib.bk_last_error().decode(errors='replace')}")


def initial_parameters(seed=0):
    """He-style initial weights for SiLU layers, zero biases (FP32 vector of PARAMS values)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    p[0:448] = rng.standard_normal(448) * np.sqrt(2.0 / FEATURES)
    p[512:4608] = rng.standard_normal(4096) * np.sqrt(2.0 / 64)
    p[4672:4864] = rng.standard_normal(192) * np.sqrt(1.0 / 64)
    return p


@dataclass
class Normalisation:
    in_mean: np.ndarray      # (7,)
    in_scale: np.ndarray     # (7,)
    out_scale: np.ndarray    # (3,)
    in_low: np.ndarray       # (7,) training range (raw units) for the out-of-distribution test
    in_high: np.ndarray

    @classmethod
    def fit(cls, features, targets, margin=0.0):
        f = np.asarray(features, np.float64)[:, :FEATURES]
        t = np.asarray(targets, np.float64)[:, :OUTPUTS]
        mean = f.mean(0)
        scale = f.std(0)
        scale[scale < 1e-12] = 1.0
        out = np.sqrt((t * t).mean(0))
        out[out < 1e-12] = 1.0
        lo, hi = f.min(0), f.max(0)
        pad = margin * (hi - lo)
        return cls(mean.astype(np.float32), scale.astype(np.float32), out.astype(np.float32),
                   (lo - pad).astype(np.float32), (hi + pad).astype(np.float32))

    def struct(self):
        s = BkMlpNorm()
        s.in_mean[:FEATURES] = [float(v) for v in self.in_mean]
        s.in_scale[:] = [float(v) for v in self.in_scale] + [1.0]
        s.out_scale[:OUTPUTS] = [float(v) for v in self.out_scale]
        s.out_scale[3] = 1.0
        return s


class ReturnMapMlp:
    """Device-resident parameters, Adam state and packed operands of the surrogate network."""

    def __init__(self, normalisation, params=None, device="cuda", seed=0):
        self.device = torch.device(device)
        self.lib = _lib_handle()
        self.norm = normalisation
        self._norm_struct = normalisation.struct()
        p = initial_parameters(seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.as_tensor(p, device=self.device).clone()
        self.grads = torch.zeros(PARAMS, dtype=torch.float32, device=self.device)
        self.m = torch.zeros_like(self.grads)
        self.v = torch.zeros_like(self.grads)
        self.step = 0
        self.packed = torch.zeros(PACKED_BYTES, dtype=torch.uint8, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss_sum = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.pack()

    def pack(self):
        _call(self.lib, "bk_mlp_pack", self.params.data_ptr(), self.packed.data_ptr(), _lib.stream_handle())

    @staticmethod
    def _rows8(x):
        x = torch.as_tensor(x, dtype=torch.float32)
        out = torch.zeros(x.shape[0], 8 if x.shape[1] <= 8 else x.shape[1], dtype=torch.float32, device=x.device)
        out[:, :x.shape[1]] = x
        return out.contiguous()

    def infer(self, features):
        """Predicted return (n, 3) for raw features (n, 7) on the device, via the tensor cores."""
        f = self._rows8(features.to(self.device))
        n = f.shape[0]
        out = torch.empty(n, 4, dtype=torch.float32, device=self.device)
        self.status.zero_()
        _call(self.lib, "bk_mlp_infer", n, f.data_ptr(), C.byref(self._norm_struct), self.packed.data_ptr(),
              out.data_ptr(), self.status.data_ptr(), _lib.stream_handle())
        if int(self.status.item()) != 0:
            raise RuntimeError("bk_mlp_infer: a tensor-core completion wait gave up")
        return out[:, :OUTPUTS]

    def gradient(self, features, targets, accumulate=False):
        """Loss gradient of one batch into self.grads; returns the batch's mean squared error (device)."""
        f = self._rows8(features.to(self.device))
        t = torch.zeros(f.shape[0], 4, dtype=torch.float32, device=self.device)
        t[:, :OUTPUTS] = torch.as_tensor(targets, dtype=torch.float32, device=self.device)[:, :OUTPUTS]
        if not accumulate:
            self.grads.zero_()
        self.loss_sum.zero_()
        _call(self.lib, "bk_mlp_gradient", f.shape[0], f.data_ptr(), t.data_ptr(), C.byref(self._norm_struct),
              self.params.data_ptr(), self.grads.data_ptr(), self.loss_sum.data_ptr(), _lib.stream_handle())
        return self.loss_sum / (f.shape[0] * OUTPUTS)

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        _call(self.lib, "bk_mlp_adam", self.grads.data_ptr(), self.params.data_ptr(), self.m.data_ptr(),
              self.v.data_ptr(), self.step, lr, beta1, beta2, eps, _lib.stream_handle())

    def train(self, features, targets, epochs=10, batch=8192, lr=2e-3, lr_final=1e-4, seed=0, log=None):
        """Adam on the mean squared error (units of out_scale) with a cosine learning-rate decay.
        ``features``/``targets`` are device tensors (n, 7) / (n, 3). Returns the per-epoch mean losses."""
        f = self._rows8(features.to(self.device))
        t = torch.as_tensor(targets, dtype=torch.float32, device=self.device)
        n = f.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        history = []
        k = 0
        for epoch in range(epochs):
            order = torch.randperm(n, device=self.device, generator=g)
            acc = torch.zeros((), dtype=torch.float64, device=self.device)
            for s in range(steps_per_epoch):
                idx = order[s * batch:(s + 1) * batch]
                acc += self.gradient(f[idx], t[idx])[0]
                rate = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(1, total - 1)))
                self.adam(float(rate))
                k += 1
            history.append(float(acc) / steps_per_epoch)
            if log:
                log(epoch, history[-1])
        self.pack()
        return history

    def state_dict(self):
        n = self.norm
        return dict(params=self.params.cpu().numpy(), in_mean=n.in_mean, in_scale=n.in_scale, out_scale=n.out_scale,
                    in_low=n.in_low, in_high=n.in_high)

    @classmethod
    def from_state_dict(cls, d, device="cuda"):
        norm = Normalisation(*(np.asarray(d[k], np.float32) for k in ("in_mean", "in_scale", "out_scale",
                                                                        "in_low", "in_high")))
        return cls(norm, params=d["params"], device=device)


def _surrogate_struct(net=None, samples=None, sample_count=None, stride=1, offset=0, judge_error=None,
                      judge_stride=0, path_counts=None):
    from .physics.substep import BkReturnSurrogate
    s = BkReturnSurrogate()
    if net is not None:
        s.packed = net.packed.data_ptr()
        s.norm = net.norm.struct()
        s.in_low[:FEATURES] = [float(v) for v in net.norm.in_low]
        s.in_high[:FEATURES] = [float(v) for v in net.norm.in_high]
    if samples is not None:
        s.samples = samples.data_ptr()
        s.sample_count = sample_count.data_ptr()
        s.sample_capacity = samples.shape[0]
        s.sample_stride, s.sample_offset = int(stride), int(offset)
    if judge_error is not None:
        s.judge_error, s.judge_stride = judge_error.data_ptr(), int(judge_stride)
    if path_counts is not None:
        s.path_counts = path_counts.data_ptr()
    return s


def _engine(sim):
    from .physics.materials.ding import DingMaterial
    if not isinstance(sim.material, DingMaterial):
        raise ValueError("the return-map surrogate needs the ding2019 material")
    return sim._engine


def _random_rotations(n, generator, device):
    """Uniform random rotations from unit quaternions (closed form, float64)."""
    q = torch.randn(n, 4, device=device, generator=generator, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1).view(n, 3, 3)


def RandomizeReturnInputs(sim, seed=0, strain=0.12, volume=0.03, temperature=(295.0, 345.0),
                          porosity=(0.05, 0.45), water_scale=(0.25, 1.75), gas_scale=(0.2, 3.0)):
    """Give every particle of ``sim``'s current state an independent random material state for
    harvesting training pairs: elastic gradient Fe = R diag(exp(e)) R^T (random rotation, deviatoric
    log strains of scale ``strain``, volumetric within +-``volume``), deformation gradient
    F = Fe (1 - n0 + n)^(1/3), porosity n, temperature, and water and gas content scaled from the
    values the simulator held at its first randomisation. The exact return map is then evaluated on
    a broad cover of its inputs."""
    eng = _engine(sim)
    st = sim.current_state
    dev = sim.device
    n = sim.particle_data.particle_count
    m = st.material_state
    base = sim._buffers.get("randomize_base")
    if base is None:
        base = dict(water=st.transport_state.water_masses.clone() if st.transport_state is not None else None,
                    gas=m.gas_moles.clone() if eng.gas else None)
        sim._buffers["randomize_base"] = base
    g = torch.Generator(device=dev).manual_seed(int(seed))
    q = _random_rotations(n, g, dev)
    e = torch.randn(n, 3, device=dev, generator=g, dtype=torch.float64) * (strain / 2)
    e = e - e.mean(1, keepdim=True) + (torch.rand(n, 1, device=dev, generator=g, dtype=torch.float64) * 2 - 1) * volume
    Fe = q @ torch.diag_embed(torch.exp(e)) @ q.transpose(1, 2)
    n0 = sim.material.ding_config.porosity
    u = lambda lo, hi: lo + (hi - lo) * torch.rand(n, device=dev, generator=g, dtype=torch.float64)  # noqa: E731
    por = u(*porosity)
    m.elastic_gradients.copy_(Fe)
    st.deformation_gradients.copy_(Fe * torch.pow(1.0 - n0 + por, 1.0 / 3.0)[:, None, None])
    st.affine_velocities.zero_()
    st.particle_velocities.zero_()
    m.porosities.copy_(por)
    m.gelled.zero_()
    T = u(*temperature)
    m.temperatures.copy_(T)
    if st.transport_state is not None:
        st.transport_state.temperatures.copy_(T)
        st.transport_state.water_masses.copy_(base["water"] * u(*water_scale))
    if eng.gas:
        m.gas_moles.copy_(base["gas"] * u(*gas_scale))


def HarvestReturnSamples(sim, steps, capacity, stride=1):
    """Run ``steps`` substeps of ``sim`` on the exact return map, keeping up to ``capacity``
    (features, return) pairs of yielding particles, every ``stride``-th particle (the sampled offset
    rotates per substep). Returns device tensors (n, 7) and (n, 3) and the number of yielding
    particle-substeps seen on the stride."""
    eng = _engine(sim)
    rows = torch.zeros(capacity, 12, dtype=torch.float32, device=sim.device)
    count = torch.zeros(1, dtype=torch.int32, device=sim.device)
    try:
        for k in range(steps):
            eng.surrogate = _surrogate_struct(samples=rows, sample_count=count, stride=stride, offset=k % stride)
            sim.AdvanceUnchecked(1)
    finally:
        eng.surrogate = None
    seen = int(count.item())
    n = min(seen, capacity)
    return rows[:n, :FEATURES].clone(), rows[:n, FEATURES:FEATURES + OUTPUTS].clone(), seen


class ReturnMapSurrogate:
    """A trained ``ReturnMapMlp`` attached to simulators: the fused G2P kernel then evaluates the
    network on the tensor cores and returns yielding in-range particles with it."""

    def __init__(self, net, judge_stride=0):
        self.net = net
        self.judge_stride = int(judge_stride)
        self.path_counts = torch.zeros(3, dtype=torch.int32, device=net.device)
        self.judge_error = torch.zeros(1, dtype=torch.float32, device=net.device)

    def attach(self, sim):
        eng = _engine(sim)
        self.net.pack()
        eng.surrogate = _surrogate_struct(net=self.net, judge_error=self.judge_error if self.judge_stride else None,
                                          judge_stride=self.judge_stride, path_counts=self.path_counts)
        return self

    @staticmethod
    def detach(sim):
        _engine(sim).surrogate = None

    def reset_statistics(self):
        self.path_counts.zero_()
        self.judge_error.zero_()

    def statistics(self):
        c = self.path_counts.tolist()
        return dict(elastic=c[0], surrogate=c[1], exact_yielding=c[2],
                    judge_max_log_strain_error=float(self.judge_error.item()) if self.judge_stride else None)


def BuildTrainingSet(sim, rounds=6, steps=3, capacity_per_round=3_000_000, seed=0):
    """Harvest (features, return) pairs from ``rounds`` randomised material states of ``sim``
    (RandomizeReturnInputs), ``steps`` exact substeps each; non-finite rows are dropped."""
    feats, targs = [], []
    for r in range(rounds):
        RandomizeReturnInputs(sim, seed=seed + r)
        f, t, _ = HarvestReturnSamples(sim, steps, capacity_per_round)
        ok = torch.isfinite(f).all(1) & torch.isfinite(t).all(1)
        feats.append(f[ok])
        targs.append(t[ok])
    return torch.cat(feats), torch.cat(targs)


def TrainReturnSurrogate(features, targets, epochs=30, batch=8192, lr=3e-3, lr_final=3e-5, validation=0.05, seed=0):
    """Fit a ReturnMapMlp on device tensors; returns (net, history, validation RMS error per output,
    validation RMS of the targets)."""
    g = torch.Generator(device=features.device).manual_seed(seed)
    perm = torch.randperm(features.shape[0], device=features.device, generator=g)
    nv = max(1, int(features.shape[0] * validation))
    fv, tv = features[perm[:nv]], targets[perm[:nv]]
    ft, tt = features[perm[nv:]], targets[perm[nv:]]
    net = ReturnMapMlp(Normalisation.fit(ft.cpu().numpy(), tt.cpu().numpy()), device=features.device, seed=seed)
    history = net.train(ft, tt, epochs=epochs, batch=batch, lr=lr, lr_final=lr_final, seed=seed)
    err = (net.infer(fv) - tv).pow(2).mean(0).sqrt()
    return net, history, err.tolist(), tv.pow(2).mean(0).sqrt().tolist()


def SaveReturnSurrogate(net, path, **metadata):
    np.savez(path, **net.state_dict(), **{k: np.asarray(v) for k, v in metadata.items()})


def LoadReturnSurrogate(path, device="cuda"):
    with np.load(path) as d:
        return ReturnMapMlp.from_state_dict({k: d[k] for k in d.files}, device=device)


def main(argv=None):
    """Harvest from the randomised box loaf (1M particles, 128^3, Ding + gas + thermal-water) and
    train the surrogate; writes the weights, normalisation and training range to ``--out``."""
    import argparse
    import time
    from . import scenes
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--out", required=True)
    p.add_argument("--particles", type=int, default=1_000_000)
    p.add_argument("--rounds", type=int, default=6)
    p.add_argument("--epochs", type=int, default=30)
    p.add_argument("--seed", type=int, default=0)
    a = p.parse_args(argv)
    t0 = time.time()
    scene = scenes.box_loaf(resolution=128, particle_count=a.particles, seed=a.seed, initial_temperature=318.15)
    sim = scenes.make_simulator(scene, diagnostics="lean")
    f, t = BuildTrainingSet(sim, rounds=a.rounds, seed=a.seed)
    t1 = time.time()
    net, history, err, rms = TrainReturnSurrogate(f, t, epochs=a.epochs, seed=a.seed)
    t2 = time.time()
    SaveReturnSurrogate(net, a.out, samples=f.shape[0], history=np.asarray(history), validation_rms_error=err,
                        target_rms=rms)
    print(f"samples {f.shape[0]} (harvest {t1 - t0:.1f} s), training {t2 - t1:.1f} s, validation RMS error {err} "
          f"of target RMS {rms}", flush=True)


if __name__ == "__main__":
    main()
