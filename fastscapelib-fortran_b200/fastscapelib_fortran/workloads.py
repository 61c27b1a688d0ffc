"""Seeded synthetic workloads for the continental time step.

The reference publishes no dataset; these generators produce inputs with the
shapes, sizes and value distributions of the benchmark configurations:

* ``plain_d8_101``: 101x101, xl=yl=100 km, h~U[0,1), interior uplift 1e-3,
  bc=1111, single flow direction (p=-2), kf=1e-5, m=0.4, n=1, kd=1e-2,
  dt=1000, 200 steps.
* ``mfd_2049``: 2049x2049, xl=yl=200 km, h=U[0,10)+1e-3*j, interior uplift
  5e-4, bc=1010 (x cyclic), multiple flow p=1.1, kf=2e-6, m=0.45, n=1.5,
  kd=5e-2, dt=500, 500 steps.
* ``closed_basin_8193``: 8193x8193, 50 m spacing, h~U[0,50), bc=0101
  (y cyclic), p=1, kf=1e-5, m=0.5, n=1, kd=1e-2, dt=200, 50 steps.
* ``uneven_d8`` (many grids at once): 256 square grids with sides drawn
  log-uniform in [129, 1025] (odd), 100 m spacing, per grid kf~logU[1e-6,1e-4],
  m~U[0.35,0.6], n~U[1,2], kd~logU[1e-3,1e-1], interior uplift U[1e-4,2e-3],
  h~U[0,1), bc=1111, single flow direction, dt=1000, 100 steps.
* ``served_mfd`` (requests): sides log-uniform in [257, 4097] (odd), steps
  uniform in 20..400, the parameters of ``mfd_2049``, each from its own seed.

Arrays are float64 in the reference layout ij = i + (j-1)*nx (x fastest),
i.e. numpy ``reshape(ny, nx)``.  Any side length can be substituted to get a
scaled version of a configuration with the same parameters.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    xl: float
    yl: float
    dt: float
    bc: int
    kf: np.ndarray
    kfsed: float
    m: float
    n: float
    kd: np.ndarray
    kdsed: float
    g1: float
    g2: float
    p: float
    u: np.ndarray
    h0: np.ndarray
    nsteps: int
    extra: dict = field(default_factory=dict)

    @property
    def nn(self) -> int:
        return self.nx * self.ny

    def job(self, **kw):
        """This workload as a batch Job (fastscapelib_fortran.Job)."""
        from . import Job
        return Job(self.nx, self.ny, self.xl, self.yl, self.dt, self.h0, self.kf, self.kd, self.u,
                   self.m, self.n, self.p, bc=self.bc, nsteps=self.nsteps, kfsed=self.kfsed,
                   kdsed=self.kdsed, g1=self.g1, g2=self.g2, **kw)

    def apply(self, api) -> None:
        """Drive a fastscape_* API module (reference-shaped) through set-up."""
        api.fastscape_init()
        api.fastscape_set_nx_ny(self.nx, self.ny)
        api.fastscape_setup()
        api.fastscape_set_xl_yl(self.xl, self.yl)
        api.fastscape_set_dt(self.dt)
        api.fastscape_init_h(self.h0.copy())
        api.fastscape_set_erosional_parameters(self.kf, self.kfsed, self.m, self.n, self.kd,
                                               self.kdsed, self.g1, self.g2, self.p)
        api.fastscape_set_u(self.u)
        api.fastscape_set_bc(self.bc)


def _interior(nx: int, ny: int, value: float) -> np.ndarray:
    u = np.full((ny, nx), value, dtype=np.float64)
    u[0, :] = 0.0
    u[-1, :] = 0.0
    u[:, 0] = 0.0
    u[:, -1] = 0.0
    return u.ravel()


def plain_d8(nx: int = 101, ny: int | None = None, seed: int = 12345, nsteps: int = 200,
             p: float = -2.0) -> Workload:
    ny = nx if ny is None else ny
    rng = np.random.default_rng(seed)
    h0 = rng.random(nx * ny)
    nn = nx * ny
    return Workload("plain_d8_%dx%d" % (nx, ny), nx, ny, 1.0e5, 1.0e5 * (ny - 1) / (nx - 1),
                    1.0e3, 1111, np.full(nn, 1.0e-5), -1.0, 0.4, 1.0, np.full(nn, 1.0e-2), -1.0,
                    0.0, 0.0, p, _interior(nx, ny, 1.0e-3), h0, nsteps)


def mfd(nx: int = 2049, ny: int | None = None, seed: int = 12345, nsteps: int = 500,
        p: float = 1.1, n: float = 1.5, bc: int = 1010) -> Workload:
    ny = nx if ny is None else ny
    rng = np.random.default_rng(seed)
    nn = nx * ny
    j = np.repeat(np.arange(ny, dtype=np.float64), nx)
    h0 = rng.random(nn) * 10.0 + 1.0e-3 * j
    dx = 2.0e5 / 2048.0
    return Workload("mfd_%dx%d" % (nx, ny), nx, ny, dx * (nx - 1), dx * (ny - 1), 500.0, bc,
                    np.full(nn, 2.0e-6), -1.0, 0.45, n, np.full(nn, 5.0e-2), -1.0, 0.0, 0.0, p,
                    _interior(nx, ny, 5.0e-4), h0, nsteps)


def closed_basin(nx: int = 8193, ny: int | None = None, seed: int = 12345,
                 nsteps: int = 50) -> Workload:
    ny = nx if ny is None else ny
    rng = np.random.default_rng(seed)
    nn = nx * ny
    h0 = rng.random(nn) * 50.0
    return Workload("closed_basin_%dx%d" % (nx, ny), nx, ny, 50.0 * (nx - 1), 50.0 * (ny - 1),
                    200.0, 101, np.full(nn, 1.0e-5), -1.0, 0.5, 1.0, np.full(nn, 1.0e-2), -1.0,
                    0.0, 0.0, 1.0, _interior(nx, ny, 5.0e-4), h0, nsteps)


def _odd_side(rng, lo: int, hi: int) -> int:
    s = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
    s += 1 - s % 2
    return max(lo, min(hi, s))


def uneven_d8(count: int = 256, seed: int = 12345, nsteps: int = 100, lo: int = 129,
              hi: int = 1025) -> list:
    """Many uneven single-flow grids (per-grid parameters drawn from `seed`,
    initial elevation of grid k from seed + k)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx = _odd_side(rng, lo, hi)
        kf = 10.0 ** rng.uniform(-6.0, -4.0)
        m = rng.uniform(0.35, 0.6)
        n = rng.uniform(1.0, 2.0)
        kd = 10.0 ** rng.uniform(-3.0, -1.0)
        up = rng.uniform(1.0e-4, 2.0e-3)
        nn = nx * nx
        h0 = np.random.default_rng(seed + k).random(nn)
        out.append(Workload("uneven_d8_%d_%dx%d" % (k, nx, nx), nx, nx, 100.0 * (nx - 1),
                            100.0 * (nx - 1), 1.0e3, 1111, np.full(nn, kf), -1.0, m, n,
                            np.full(nn, kd), -1.0, 0.0, 0.0, -2.0, _interior(nx, nx, up), h0,
                            nsteps))
    return out


def served_mfd(count: int, seed: int = 12345, lo: int = 257, hi: int = 4097,
               steps: tuple = (20, 400)) -> list:
    """Requests of the served configuration: multiple-flow grids with the
    parameters of ``mfd``, uneven sizes and step counts."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx = _odd_side(rng, lo, hi)
        ns = int(rng.integers(steps[0], steps[1] + 1))
        out.append(mfd(nx, seed=seed + 1 + k, nsteps=ns))
    return out
