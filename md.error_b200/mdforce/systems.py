"""Seeded synthetic systems of the benchmark workloads.

  lj_fluid_fcc     4000-atom fcc LJ fluid, L = 16.796 (rho* = 0.8442), +-0.05 jitter
  charged_fluid    20736 +-1 charges in a 30^3 box, 0.8 sigma minimum separation
  lj_slab          65536-atom liquid-vapour slab in 40 x 40 x 160: liquid rho* = 0.78
                   for |z - 80| < 24.84, vapour rho* = 0.02 elsewhere (the slab is
                   widened from 20 sigma so that both densities and N = 65536 hold)
  charged_slab     1048576 +-1 charges in 100 x 100 x 400: liquid 0.8 for |z - 200| < 64,
                   vapour count trimmed so N = 2^20
All generation is host code in libmdforce (md_synth_*), seeded with mt19937_64.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import lib
from .core import check, _p


@dataclass
class SyntheticSystem:
    name: str
    pos: np.ndarray
    box: np.ndarray
    vel: np.ndarray = None
    charge: np.ndarray = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.pos.shape[0]


def fcc(cells, box, jitter, seed):
    box = np.asarray(box, np.float64)
    n = 4 * cells[0] * cells[1] * cells[2]
    pos = np.empty((n, 3), np.float64)
    check(lib.md_synth_fcc(cells[0], cells[1], cells[2], _p(box), jitter, seed, _p(pos)), "md_synth_fcc")
    return pos


def slab(n, n_in, box, axis, center, half_width, min_sep, seed):
    box = np.asarray(box, np.float64)
    pos = np.empty((n, 3), np.float64)
    check(lib.md_synth_slab(n, n_in, _p(box), axis, center, half_width, min_sep, seed, _p(pos)),
          "md_synth_slab")
    return pos


def maxwell(n, temperature, seed, mass=None):
    vel = np.empty((n, 3), np.float64)
    m = None if mass is None else _p(np.ascontiguousarray(mass, np.float64))
    check(lib.md_synth_maxwell(n, m, temperature, seed, _p(vel)), "md_synth_maxwell")
    return vel


def charges(n, seed):
    q = np.empty(n, np.float64)
    check(lib.md_synth_charges(n, seed, _p(q)), "md_synth_charges")
    return q


def lj_fluid_fcc(cells=10, L=16.796, jitter=0.05, temperature=1.0, seed=0):
    box = np.array([L, L, L])
    pos = fcc((cells, cells, cells), box, jitter, seed)
    vel = maxwell(pos.shape[0], temperature, seed + 1)
    return SyntheticSystem("lj_fluid_fcc", pos, box, vel,
                           meta=dict(rc=2.5, skin=0.3, dt=0.005, gamma=0.1, T=temperature))


def charged_fluid(n=20736, L=30.0, min_sep=0.8, seed=0):
    box = np.array([L, L, L])
    pos = slab(n, n, box, 2, 0.5 * L, 0.5 * L + 1.0, min_sep, seed)
    q = charges(n, seed + 7)
    return SyntheticSystem("charged_fluid", pos, box, None, q,
                           meta=dict(rc=3.0, beta=0.95, mesh=(64, 64, 64), order=6))


def slab_counts(n, box, axis, rho_l, rho_v):
    """Liquid thickness and atom counts so that both densities hold with N = n."""
    area = box[0] * box[1] * box[2] / box[axis]
    Lz = box[axis]
    thick = (n - rho_v * area * Lz) / ((rho_l - rho_v) * area)
    n_in = int(round(rho_l * area * thick))
    return thick, n_in


def lj_slab(n=65536, box=(40.0, 40.0, 160.0), rho_l=0.78, rho_v=0.02, min_sep=0.8,
            temperature=0.85, seed=0):
    box = np.asarray(box, np.float64)
    thick, n_in = slab_counts(n, box, 2, rho_l, rho_v)
    pos = slab(n, n_in, box, 2, 0.5 * box[2], 0.5 * thick, min_sep, seed)
    vel = maxwell(n, temperature, seed + 1)
    return SyntheticSystem("lj_slab", pos, box, vel,
                           meta=dict(liquid_half_width=0.5 * thick, n_liquid=n_in, T=temperature,
                                     rc_min=2.5, rc_max=5.0, rc_step=0.5, skin=0.3, dt=0.005))


def charged_slab(n=1 << 20, box=(100.0, 100.0, 400.0), rho_l=0.8, half=64.0, min_sep=0.8,
                 seed=0):
    box = np.asarray(box, np.float64)
    n_in = int(round(rho_l * box[0] * box[1] * 2 * half))
    n_in = min(n_in, n)
    pos = slab(n, n_in, box, 2, 0.5 * box[2], half, min_sep, seed)
    q = charges(n, seed + 7)
    return SyntheticSystem("charged_slab", pos, box, None, q,
                           meta=dict(n_liquid=n_in, mesh=(128, 128, 512), order=6))
