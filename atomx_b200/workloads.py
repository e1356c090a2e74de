"""Seeded synthetic ions for the R^k engine (host-side input generation).

Each ion is a radial basis plus a set of relativistic spinors given by their
B-spline coefficients.  The spinors are the lowest positive-energy
Dirac-Coulomb eigenvectors of a kinetically balanced basis, optionally
rotated within each kappa by a seeded orthogonal matrix, so that the pair
densities are realistic (sign-changing, multi-scale) while the inputs stay
fully reproducible.  No external dataset is involved.

Named workloads (sizes as the benchmark quotes them):

* ``neon_small``      Z=10, 40 splines of order 7, r in [1e-5, 40], 7 nodes per
                      cell (N=238); 1s, 2s, 2p1/2, 2p3/2; k <= 2.
* ``ytterbium_scaleup`` Z=70, 120 splines of order 9, r in [1e-6, 60], 8 nodes
                      per cell (N=896); 200 spinors over kappa = +-1..+-7 with
                      seeded rotations; k <= 12.
* ``uneven_batch``    64 ions, Z~U{20..83}, 40..160 splines of order 7 or 9,
                      r in [1e-5, 40], ng = order; 20..150 spinors over
                      kappa = +-1..+-6; k <= 2 l_max.
* ``serving_requests`` Poisson stream (rate 200/s) of ions with Z~U{2..92},
                      30..200 splines of order 9, r in [1e-6, 60], ng = 8,
                      10..300 spinors over kappa = +-1..+-7, k_max~U{2..14}.
* ``xenon_ci_table``  Z=54, 200 splines of order 9, r in [1e-6, 60], 11 nodes
                      per cell (N=2112); 300 spinors over kappa = +-1..+-9;
                      k <= 16.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np

from . import basis as _basis
from . import dirac as _dirac

__all__ = ["IonSpec", "Ion", "build_ion", "neon_small", "ytterbium_scaleup", "uneven_batch",
           "serving_requests", "xenon_ci_table", "kappa_ladder"]


def kappa_ladder(kmax_abs: int) -> list[int]:
    """kappa order -1, +1, -2, +2, ..., -kmax_abs, +kmax_abs."""
    out: list[int] = []
    for a in range(1, kmax_abs + 1):
        out += [-a, a]
    return out


def _spread(total: int, kappas: list[int]) -> tuple[tuple[int, int], ...]:
    """Distribute ``total`` spinors over kappas, earlier kappas first."""
    base, extra = divmod(total, len(kappas))
    return tuple((kap, base + (1 if i < extra else 0)) for i, kap in enumerate(kappas)
                 if base + (1 if i < extra else 0) > 0)


@dataclass(frozen=True)
class IonSpec:
    Z: float
    ns: int
    ks: int
    n_gauss: int
    r_min: float
    r_max: float
    shells: tuple  # ((kappa, count), ...) in orbital order
    k_max: int
    seed: int | None = None  # None: unrotated eigenvectors
    name: str = ""

    @property
    def n_orbitals(self) -> int:
        return int(sum(c for _, c in self.shells))

    @property
    def nv(self) -> int:
        return self.ns - self.ks + 1

    @property
    def n_points(self) -> int:
        return self.nv * self.n_gauss


@dataclass
class Ion:
    spec: IonSpec
    bsp: dict
    P: np.ndarray  # (n_orb, ns) large-component coefficients (zero padded)
    Q: np.ndarray  # (n_orb, ns) small-component coefficients
    kappa: np.ndarray  # (n_orb,) int
    extra: dict = field(default_factory=dict)

    @property
    def n_orbitals(self) -> int:
        return int(self.P.shape[0])

    def coefficient_digest(self) -> str:
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(self.P).tobytes())
        h.update(np.ascontiguousarray(self.Q).tobytes())
        h.update(np.ascontiguousarray(self.kappa.astype(np.int64)).tobytes())
        return h.hexdigest()


def build_ion(spec: IonSpec) -> Ion:
    """Basis, spinors and kappa labels for one ion (deterministic)."""
    t = _basis.make_exponential_knots(spec.ns, spec.ks, spec.r_min, spec.r_max)
    bsp = _basis.prepare_bspline_data(t, spec.ns, spec.ks, n_gauss=spec.n_gauss, kinetic_balance=True)
    rng = np.random.default_rng(spec.seed) if spec.seed is not None else None
    Ps, Qs, kap = [], [], []
    for kappa, count in spec.shells:
        if rng is None:
            P, Q, _ = _dirac.dirac_spinors(bsp, kappa, spec.Z, count)
        else:
            P, Q = _dirac.rotated_spinors(bsp, kappa, spec.Z, count, rng)
        Ps.append(P)
        Qs.append(Q)
        kap += [kappa] * count
    return Ion(spec=spec, bsp=bsp, P=np.concatenate(Ps), Q=np.concatenate(Qs),
               kappa=np.asarray(kap, dtype=np.int64))


def neon_small() -> IonSpec:
    return IonSpec(Z=10, ns=40, ks=7, n_gauss=7, r_min=1e-5, r_max=40.0,
                   shells=((-1, 2), (1, 1), (-2, 1)), k_max=2, seed=None, name="neon_small")


def ytterbium_scaleup(seed: int = 2026) -> IonSpec:
    kaps = kappa_ladder(7)
    shells = tuple((kap, 15 if i < 4 else 14) for i, kap in enumerate(kaps))
    return IonSpec(Z=70, ns=120, ks=9, n_gauss=8, r_min=1e-6, r_max=60.0, shells=shells,
                   k_max=12, seed=seed, name="ytterbium_scaleup")


def xenon_ci_table(seed: int = 2054) -> IonSpec:
    return IonSpec(Z=54, ns=200, ks=9, n_gauss=11, r_min=1e-6, r_max=60.0,
                   shells=_spread(300, kappa_ladder(9)), k_max=16, seed=seed, name="xenon_ci_table")


def uneven_batch(seed: int = 3064, n_ions: int = 64) -> list[IonSpec]:
    rng = np.random.default_rng(seed)
    out = []
    kaps = kappa_ladder(6)
    for i in range(n_ions):
        Z = int(rng.integers(20, 84))
        ns = int(rng.integers(40, 161))
        ks = int(rng.choice([7, 9]))
        norb = int(rng.integers(20, 151))
        shells = _spread(norb, kaps)
        lmax = max(abs(k) if k > 0 else -k - 1 for k, _ in shells)
        out.append(IonSpec(Z=Z, ns=ns, ks=ks, n_gauss=ks, r_min=1e-5, r_max=40.0, shells=shells,
                           k_max=2 * lmax, seed=int(rng.integers(0, 2**31)), name=f"batch_ion{i}"))
    return out


def serving_requests(seed: int = 4200, n_requests: int = 64, rate_per_s: float = 200.0, max_ns: int = 200,
                     max_orbitals: int = 300, max_kmax: int = 14):
    """(arrival_time_s, IonSpec) pairs of a seeded Poisson request stream.

    Defaults are the serving workload (Z 2..92, 30..200 B-splines, 10..300
    spinors, k_max 2..14, sized as the Z=70 ion); the max_* arguments clip the
    ranges for small test streams.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    kaps = kappa_ladder(7)
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate_per_s))
        Z = int(rng.integers(2, 93))
        ns = int(rng.integers(30, max_ns + 1))
        norb = int(rng.integers(10, max_orbitals + 1))
        kmax = int(rng.integers(2, max_kmax + 1))
        out.append((t, IonSpec(Z=Z, ns=ns, ks=9, n_gauss=8, r_min=1e-6, r_max=60.0,
                               shells=_spread(norb, kaps), k_max=kmax,
                               seed=int(rng.integers(0, 2**31)), name=f"request{i}")))
    return out
