"""Seeded synthetic filterbanks with the shapes and value distributions of the
benchmark configurations (no public dataset is involved).

Input format (reference src/clib/dedisp.h:336-345): time-major rows of
``nchans * nbits / 8`` bytes, channels packed LSB-first. Pulses are injected
with the cold-plasma delay ``4.148808e3 * DM * (f^-2 - f_top^-2)`` seconds
(deliberately not the 4.15e3 constant of the reference delay table), rounded
to samples, with a Gaussian profile of standard deviation ``width``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

KDM = 4.148808e3  # s MHz^2 pc^-1 cm^3


@dataclass
class Pulse:
    dm: float
    t0: float        # arrival time at f_top, seconds
    width: float     # Gaussian sigma, seconds
    amp: float       # peak amplitude in input units (before quantisation)


@dataclass
class Config:
    name: str
    nchans: int
    f_top: float
    df: float
    dt: float
    nsamps: int
    nbits: int
    mean: float
    sigma: float
    pulses: List[Pulse] = field(default_factory=list)
    dm_list: Optional[np.ndarray] = None          # explicit list, or
    dm_gen: Optional[Tuple[float, float, float, float]] = None  # (start, end, ti, tol)
    seed: int = 0
    float_input: bool = False


def pulse_delays(cfg: Config, dm: float) -> np.ndarray:
    """Per-channel arrival offset (samples, rounded) of a pulse at DM."""
    f = cfg.f_top + np.arange(cfg.nchans) * cfg.df
    return np.rint(KDM * dm * (f ** -2.0 - cfg.f_top ** -2.0) / cfg.dt).astype(np.int64)


def quantise(x: np.ndarray, nbits: int) -> np.ndarray:
    return np.clip(np.rint(x), 0, (1 << nbits) - 1).astype(np.uint8)


def pack(samples: np.ndarray, nbits: int) -> np.ndarray:
    """[nsamps][nchans] values < 2^nbits -> packed bytes [nsamps][nchans*nbits/8]."""
    nsamps, nchans = samples.shape
    if nbits == 8:
        return np.ascontiguousarray(samples.astype(np.uint8))
    if nbits == 16:
        return np.ascontiguousarray(samples.astype("<u2")).view(np.uint8).reshape(nsamps, -1)
    if nbits == 32:
        return np.ascontiguousarray(samples.astype("<u4")).view(np.uint8).reshape(nsamps, -1)
    per = 8 // nbits
    v = samples.astype(np.uint8).reshape(nsamps, nchans // per, per)
    out = np.zeros((nsamps, nchans // per), np.uint8)
    for i in range(per):
        out |= (v[:, :, i] << (i * nbits)).astype(np.uint8)
    return out


def unpack(packed: np.ndarray, nbits: int, nchans: int) -> np.ndarray:
    nsamps = packed.shape[0]
    if nbits == 8:
        return packed[:, :nchans].astype(np.uint32)
    if nbits == 16:
        return packed.view("<u2").reshape(nsamps, -1)[:, :nchans].astype(np.uint32)
    if nbits == 32:
        return packed.view("<u4").reshape(nsamps, -1)[:, :nchans].astype(np.uint32)
    per = 8 // nbits
    out = np.zeros((nsamps, nchans), np.uint32)
    m = (1 << nbits) - 1
    for i in range(per):
        out[:, i::per] = (packed[:, : nchans // per] >> (i * nbits)) & m
    return out


def make_input(cfg: Config) -> np.ndarray:
    """numpy generator (small and medium sizes): packed bytes, or float32
    bytes for float_input configurations."""
    rng = np.random.default_rng(cfg.seed)
    x = rng.standard_normal((cfg.nsamps, cfg.nchans), dtype=np.float32) * cfg.sigma + cfg.mean
    for p in cfg.pulses:
        d = pulse_delays(cfg, p.dm)
        centre = p.t0 / cfg.dt + d
        half = int(np.ceil(5 * p.width / cfg.dt)) + 1
        for c in range(cfg.nchans):
            lo = max(0, int(centre[c]) - half)
            hi = min(cfg.nsamps, int(centre[c]) + half + 1)
            if lo >= hi:
                continue
            t = np.arange(lo, hi)
            x[lo:hi, c] += p.amp * np.exp(-0.5 * ((t - centre[c]) * cfg.dt / p.width) ** 2)
    if cfg.float_input:
        return np.ascontiguousarray(x.astype("<f4")).view(np.uint8).reshape(cfg.nsamps, -1)
    return pack(quantise(x, cfg.nbits), cfg.nbits)


def make_input_torch(cfg: Config, device="cuda", chunk_rows: int = 1 << 17):
    """Device generator for production sizes (torch on the GPU). Returns a
    uint8 tensor [nsamps][row_bytes] on `device`."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(cfg.seed)
    row_bytes = cfg.nchans * (32 if cfg.float_input else cfg.nbits) // 8
    out = torch.empty((cfg.nsamps, row_bytes), dtype=torch.uint8, device=device)
    delays = [(p, torch.as_tensor(pulse_delays(cfg, p.dm), device=device)) for p in cfg.pulses]
    per = 8 // cfg.nbits if cfg.nbits < 8 else 1
    shifts = torch.arange(per, device=device, dtype=torch.int32) * cfg.nbits
    for r0 in range(0, cfg.nsamps, chunk_rows):
        r1 = min(cfg.nsamps, r0 + chunk_rows)
        x = torch.randn((r1 - r0, cfg.nchans), generator=g, device=device, dtype=torch.float32)
        x.mul_(cfg.sigma).add_(cfg.mean)
        t = torch.arange(r0, r1, device=device, dtype=torch.float32)[:, None]
        for p, d in delays:
            centre = p.t0 / cfg.dt + d.to(torch.float32)[None, :]
            half = 5 * p.width / cfg.dt + 1
            near = (t - centre).abs() <= half
            if bool(near.any()):
                x.add_(torch.where(near, p.amp * torch.exp(
                    -0.5 * ((t - centre) * cfg.dt / p.width) ** 2), torch.zeros_like(x)))
        if cfg.float_input:
            out[r0:r1] = x.contiguous().view(torch.uint8).reshape(r1 - r0, row_bytes)
            continue
        q = x.round_().clamp_(0, (1 << cfg.nbits) - 1).to(torch.int32)
        if cfg.nbits == 8:
            out[r0:r1] = q.to(torch.uint8)
        elif cfg.nbits < 8:
            q = q.reshape(r1 - r0, cfg.nchans // per, per)
            out[r0:r1] = (q << shifts).sum(dim=2).to(torch.uint8)
        else:
            raise ValueError("torch generator supports nbits <= 8")
        del x, q
    return out


# ---------------------------------------------------------------------------
# The benchmark configurations
# ---------------------------------------------------------------------------

def config0(seed: int = 20261203) -> Config:
    """Plain brute-force TDD, CPU-runnable: 1024 ch, 65536 x 8-bit, 512 DMs."""
    return Config("tdd-1024ch-65536s-8bit-512dm", 1024, 1581.8, -0.390625, 250e-6, 65536, 8,
                  128.0, 16.0, [Pulse(250.0, 4.0, 1e-3, 48.0)],
                  dm_list=(500.0 * np.arange(512) / 511.0).astype(np.float32), seed=seed)


# Quantisation scale per width (noise sigma in levels, centred at mid-scale).
QSIGMA = {2: 1.0, 4: 3.0, 8: 24.0}


def config1(nbits: int = 8, seed: int = 20261204, nsamps: int = 1 << 21) -> Config:
    """Production TDD: 4096 ch, 2^21 samples, nbits in {2,4,8}, DM list
    generate_dm_list(0, 2000, 40 us, 1.25) (3643 DMs)."""
    rng = np.random.default_rng(seed)
    sig = QSIGMA[nbits]
    pulses = [Pulse(float(rng.uniform(20, 1900)), float(rng.uniform(1.0, nsamps * 64e-6 - 3.0)),
                    float(rng.uniform(0.2e-3, 5e-3)), float(rng.uniform(2, 6)) * sig)
              for _ in range(8)]
    return Config(f"tdd-4096ch-{nsamps}s-{nbits}bit", 4096, 1500.0, -0.078125, 64e-6, nsamps,
                  nbits, (2 ** nbits - 1) / 2.0, sig, pulses, dm_gen=(0.0, 2000.0, 40.0, 1.25),
                  seed=seed)


def config2(seed: int = 20261205, nsamps: int = 1 << 20) -> Config:
    """FDD: 1024 ch, 2^20 float32 N(0,1) samples, 5 pulses, 2048 DMs over
    0-1000, segmented with 2^15-sample segments."""
    rng = np.random.default_rng(seed)
    pulses = [Pulse(float(rng.uniform(50, 900)), float(rng.uniform(1.0, nsamps * 250e-6 - 5.0)),
                    2e-3, 0.5) for _ in range(5)]
    return Config("fdd-1024ch-2^20s-f32-2048dm", 1024, 1581.8, -0.390625, 250e-6, nsamps, 32,
                  0.0, 1.0, pulses,
                  dm_list=(1000.0 * np.arange(2048) / 2047.0).astype(np.float32), seed=seed,
                  float_input=True)


def config3(seed: int = 20261206, nbeams: int = 96, nsamp_range: Tuple[int, int] = (1 << 17, 1 << 20),
            dm_max_range: Tuple[float, float] = (500.0, 3000.0),
            ndm_range: Tuple[int, int] = (1024, 4096)) -> List[Config]:
    """Batched multi-beam TDD: `nbeams` beams of 1536 ch (f_top 1670 MHz,
    df -0.25 MHz, dt 81.92 us), 8-bit noise round(N(128, 16)); per beam a
    seeded nsamp, maximum DM and linear DM-trial count, and 3 pulses."""
    rng = np.random.default_rng(seed)
    beams = []
    for b in range(nbeams):
        ns = int(rng.integers(nsamp_range[0], nsamp_range[1] + 1))
        dm_max = float(rng.uniform(*dm_max_range))
        ndm = int(rng.integers(ndm_range[0], ndm_range[1] + 1))
        dur = ns * 81.92e-6
        pulses = [Pulse(float(rng.uniform(20.0, 0.9 * dm_max)), float(rng.uniform(0.05, 0.6) * dur),
                        float(rng.uniform(0.5e-3, 3e-3)), float(rng.uniform(24.0, 64.0)))
                  for _ in range(3)]
        beams.append(Config(f"beam{b:02d}-1536ch-{ns}s-{ndm}dm", 1536, 1670.0, -0.25, 81.92e-6, ns, 8,
                            128.0, 16.0, pulses,
                            dm_list=(dm_max * np.arange(ndm) / max(ndm - 1, 1)).astype(np.float32),
                            seed=seed + 1 + b))
    return beams
