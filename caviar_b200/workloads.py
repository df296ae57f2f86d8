"""Seeded synthetic MD systems (the reference's benchmark shapes).

No dataset is involved anywhere: every state is generated from a seed, with the
sizes, densities and temperatures of the configurations the hot path is
measured on.  Units are reduced LJ units (epsilon = sigma = m = k_b = 1), as in
the reference (`src/caviar/objects/force_field/lj.cpp`, `atom_data.cpp:121-126`).

`MDSystem` carries one periodic system: the box (`domain box`), per-type mass
and charge (`atom_data add_type_mass / add_type_charge`), the atoms, and the
settings of the reference objects on the hot path (`neighborlist basic`,
`force_field lj`, `force_field electrostatic_ewald_r`,
`force_field electrostatic_ewald_k`, `md_simulator basic`).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


@dataclasses.dataclass
class LJParams:
    """force_field lj: cutoff, per-type-pair epsilon/sigma, optional cutoff_list."""
    cutoff: float
    epsilon: np.ndarray  # (T, T)
    sigma: np.ndarray  # (T, T)
    cutoff_list: Optional[np.ndarray] = None  # (T, T) or None
    ignore_intra_molecule: bool = False
    jump_tol: float = 0.0  # > 0 enables the reference's jump_tol clamp


@dataclasses.dataclass
class EwaldRParams:
    """force_field electrostatic_ewald_r: alpha, k_electrostatic.

    cutoff < 0 keeps the reference's behaviour: every Verlet-list pair is
    summed (electrostatic_ewald_r.cpp:142-226 has no cutoff test)."""
    alpha: float
    k_electrostatic: float = 1.0
    cutoff: float = -1.0
    lam: Optional[np.ndarray] = None  # (T, T) same-molecule scaling, or None


@dataclasses.dataclass
class EwaldKParams:
    """force_field electrostatic_ewald_k: alpha, k_max per axis, k_electrostatic."""
    alpha: float
    kmax: tuple
    k_electrostatic: float = 1.0


@dataclasses.dataclass
class MDSystem:
    lo: np.ndarray
    hi: np.ndarray
    mass: np.ndarray  # (T,)
    charge: np.ndarray  # (T,)
    pos: np.ndarray  # (N, 3) float64
    vel: np.ndarray  # (N, 3) float64
    type: np.ndarray  # (N,) int32
    cutoff: float  # neighborlist cutoff
    coef: float  # neighborlist cutoff_extra_coef
    ghost_cutoff: float  # atom_data ghost_cutoff
    dt: float
    bc: tuple = (1, 1, 1)
    mol: Optional[np.ndarray] = None  # (N,) int32 molecule index, -1 = none
    lj: Optional[LJParams] = None
    ewald_r: Optional[EwaldRParams] = None
    ewald_k: Optional[EwaldKParams] = None
    k_b: float = 1.0
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_types(self) -> int:
        return int(len(self.mass))

    @property
    def box(self) -> np.ndarray:
        return np.asarray(self.hi, np.float64) - np.asarray(self.lo, np.float64)

    def copy(self) -> "MDSystem":
        return dataclasses.replace(self, pos=self.pos.copy(), vel=self.vel.copy(), type=self.type.copy(),
                                   mol=None if self.mol is None else self.mol.copy())


def maxwell_boltzmann(n: int, temperature: float, rng: np.random.Generator, mass: float = 1.0) -> np.ndarray:
    """Gaussian velocities, centre-of-mass motion removed, rescaled so that
    2 KE / (3N - 3) = T (the reference's periodic dof, kinetic_energy.cpp:646-718)."""
    v = rng.normal(0.0, np.sqrt(temperature / mass), size=(n, 3))
    v -= v.mean(axis=0)
    ke = 0.5 * mass * np.sum(v * v)
    t_now = 2.0 * ke / (3 * n - 3)
    if t_now > 0:
        v *= np.sqrt(temperature / t_now)
    return v


def fcc_lattice(ncell: int, density: float, temperature: float, seed: int, cutoff: float = 2.5,
                skin: float = 0.3, dt: float = 0.005, jitter: float = 0.0) -> MDSystem:
    """Plain LJ fluid on an FCC lattice (4 atoms per cubic cell) in a periodic
    cube, epsilon = sigma = m = 1, lattice offset a/4 from the faces.  jitter > 0
    displaces every atom uniformly in [-jitter, jitter]^3 (a perfect lattice has
    zero net forces, which makes a poor force test)."""
    a = (4.0 / density) ** (1.0 / 3.0)
    L = ncell * a
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], np.float64)
    g = np.arange(ncell, dtype=np.float64)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = ((cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) + 0.25) * a
    n = pos.shape[0]
    rng = np.random.default_rng(seed)
    vel = maxwell_boltzmann(n, temperature, rng)
    if jitter > 0:
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    coef = (cutoff + skin) / cutoff
    lj = LJParams(cutoff=cutoff, epsilon=np.ones((1, 1)), sigma=np.ones((1, 1)))
    return MDSystem(lo=np.zeros(3), hi=np.full(3, L), mass=np.ones(1), charge=np.zeros(1), pos=pos, vel=vel,
                    type=np.zeros(n, np.int32), cutoff=cutoff, coef=coef, ghost_cutoff=cutoff * coef, dt=dt,
                    lj=lj, name=f"fcc{ncell}_N{n}")


def random_ions(n: int, box: float, seed: int, min_sep: float = 0.9, temperature: float = 1.0,
                lj_cutoff: float = 2.5, alpha: float = 0.3, rc: float = 10.0, coef: float = 1.03,
                kmax: int = 8, dt: float = 0.005) -> MDSystem:
    """Charged LJ electrolyte: n ions alternating type 0 (q=+1) / type 1 (q=-1),
    uniform in a periodic cube with a minimum separation (cell-grid
    rejection), Gaussian velocities at T with COM removed.

    The neighbour list is sized for the Ewald real-space cutoff rc (the larger
    one); LJ keeps its own 2.5 sigma cutoff test on that list."""
    rng = np.random.default_rng(seed)
    ncell = max(1, int(np.floor(box / min_sep)))
    w = box / ncell
    grid: dict = {}
    pos = np.empty((n, 3))
    k = 0
    ms2 = min_sep * min_sep
    while k < n:
        p = rng.uniform(0.0, box, size=3)
        c = tuple(int(x) for x in np.minimum((p / w).astype(np.int64), ncell - 1))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    q = ((c[0] + dx) % ncell, (c[1] + dy) % ncell, (c[2] + dz) % ncell)
                    for j in grid.get(q, ()):
                        d = p - pos[j]
                        d -= box * np.round(d / box)
                        if d @ d < ms2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pos[k] = p
            grid.setdefault(c, []).append(k)
            k += 1
    vel = rng.normal(0.0, np.sqrt(temperature), size=(n, 3))
    vel -= vel.mean(axis=0)
    typ = (np.arange(n) % 2).astype(np.int32)
    lj = LJParams(cutoff=lj_cutoff, epsilon=np.ones((2, 2)), sigma=np.ones((2, 2)))
    er = EwaldRParams(alpha=alpha, k_electrostatic=1.0)
    ek = EwaldKParams(alpha=alpha, kmax=(kmax, kmax, kmax), k_electrostatic=1.0)
    return MDSystem(lo=np.zeros(3), hi=np.full(3, box), mass=np.ones(2), charge=np.array([1.0, -1.0]), pos=pos,
                    vel=vel, type=typ, cutoff=rc, coef=coef, ghost_cutoff=rc * coef, dt=dt, lj=lj, ewald_r=er,
                    ewald_k=ek, name=f"ions_N{n}_L{box:g}")


def config_lj_4000(seed: int = 1, jitter: float = 0.0) -> MDSystem:
    """4000 LJ atoms, FCC 10^3 cells, rho* = 0.8442, T* = 0.72, rc 2.5, skin 0.3, dt 0.005
    (jitter > 0 displaces the lattice sites, for force checks away from the
    perfect lattice, where every force vanishes)."""
    return fcc_lattice(10, 0.8442, 0.72, seed, jitter=jitter)


def config_ions_8000(seed: int = 2) -> MDSystem:
    """8000 ions (+-1) in L = 40, LJ rc 2.5, Ewald alpha 0.3, rc 10 (skin 0.3), kmax 8, T* = 1."""
    return random_ions(8000, 40.0, seed)


def config_lj_1m(seed: int = 3, jitter: float = 0.0) -> MDSystem:
    """1,048,576 LJ atoms, FCC 64^3 cells, rho* = 0.8442, T* = 0.72, rc 2.5, skin 0.3
    (jitter as in config_lj_4000)."""
    return fcc_lattice(64, 0.8442, 0.72, seed, jitter=jitter)


@dataclasses.dataclass
class ReplicaBatch:
    """Many small periodic LJ + charge replicas (one system per box)."""
    n: np.ndarray  # (R,) atoms per replica
    box: np.ndarray  # (R,) cube edge
    pos: np.ndarray  # (sum n, 3), replica order
    vel: np.ndarray
    type: np.ndarray  # 0 neutral, 1 q=+1, 2 q=-1
    temperature: np.ndarray  # (R,)
    rc_lj: np.ndarray
    rc_r: np.ndarray
    mass: np.ndarray = dataclasses.field(default_factory=lambda: np.ones(3))
    charge: np.ndarray = dataclasses.field(default_factory=lambda: np.array([0.0, 1.0, -1.0]))
    epsilon: np.ndarray = dataclasses.field(default_factory=lambda: np.ones((3, 3)))
    sigma: np.ndarray = dataclasses.field(default_factory=lambda: np.ones((3, 3)))
    alpha: float = 0.35
    kmax: int = 6
    k_e: float = 1.0
    dt: float = 0.005

    @property
    def offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.n)])


def replica_batch(n_rep: int = 1024, seed: int = 4, n_min: int = 64, n_max: int = 2048, density: float = 0.8,
                  lj_cutoff: float = 2.5, sizes=None) -> ReplicaBatch:
    """n_rep replicas, atom counts uniform in [n_min, n_max], rho* = 0.8, half
    the atoms charged +-1 (net neutral), T uniform in [0.7, 1.5].  Atoms start
    on a simple-cubic grid (random subset of sites, small jitter).  Cutoffs:
    LJ min(2.5, L/2); Ewald real space L/2 (the minimum image; every box here
    is smaller than twice a 9-sigma real-space cutoff).  sizes, when given,
    fixes the atom counts (and n_rep)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, size=n_rep) if sizes is None else np.asarray(sizes, np.int64)
    boxes = (ns / density) ** (1.0 / 3.0)
    pos, vel, typ = [], [], []
    temps = rng.uniform(0.7, 1.5, size=len(ns))
    for n, L, T in zip(ns, boxes, temps):
        m = int(np.ceil(n ** (1.0 / 3.0)))
        g = (np.arange(m) + 0.5) * (L / m)
        sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
        p = sites[rng.choice(len(sites), size=n, replace=False)]
        p = (p + rng.uniform(-0.05, 0.05, size=p.shape)) % L
        t = np.zeros(n, np.int32)
        nq = (n // 2) // 2
        idx = rng.permutation(n)
        t[idx[:nq]] = 1
        t[idx[nq:2 * nq]] = 2
        v = maxwell_boltzmann(n, T, rng)
        pos.append(p)
        vel.append(v)
        typ.append(t)
    return ReplicaBatch(n=ns.astype(np.int64), box=boxes, pos=np.concatenate(pos), vel=np.concatenate(vel),
                        type=np.concatenate(typ), temperature=temps, rc_lj=np.minimum(lj_cutoff, boxes / 2),
                        rc_r=boxes / 2)


def replica_system(b: ReplicaBatch, r: int) -> MDSystem:
    """Replica r as a system the reference's own objects can run: neighbour
    list radius = ghost cutoff = L/2 with cutoff_extra_coef 1 (the largest
    radius its one-ghost-image scheme allows, so its Ewald real-space sum,
    which has no cutoff of its own, covers the replica's minimum-image pairs
    within L/2; the list is rebuilt every step), LJ up to rc_lj, Ewald alpha
    and k_max as the batch."""
    o = b.offsets
    sl = slice(int(o[r]), int(o[r + 1]))
    L = float(b.box[r])
    T = len(b.mass)
    return MDSystem(lo=np.zeros(3), hi=np.full(3, L), mass=np.asarray(b.mass, np.float64),
                    charge=np.asarray(b.charge, np.float64), pos=b.pos[sl].copy(), vel=b.vel[sl].copy(),
                    type=b.type[sl].astype(np.int32), cutoff=0.5 * L, coef=1.0, ghost_cutoff=0.5 * L, dt=b.dt,
                    lj=LJParams(cutoff=float(b.rc_lj[r]), epsilon=np.asarray(b.epsilon).reshape(T, T),
                                sigma=np.asarray(b.sigma).reshape(T, T)),
                    ewald_r=EwaldRParams(alpha=b.alpha, k_electrostatic=b.k_e),
                    ewald_k=EwaldKParams(alpha=b.alpha, kmax=(b.kmax, b.kmax, b.kmax), k_electrostatic=b.k_e),
                    name=f"replica{r}_N{int(b.n[r])}")


@dataclasses.dataclass
class AdjointSystem:
    """One periodic cube for the trajectory adjoint: LJ + Ewald (explicit
    real-space cutoff, minimum image), parameters per type."""
    box: float
    pos: np.ndarray  # (N, 3)
    vel: np.ndarray
    type: np.ndarray  # (N,) int32
    mass: np.ndarray  # (T,)
    charge: np.ndarray  # (T,)
    epsilon: np.ndarray  # (T, T) symmetric
    sigma: np.ndarray  # (T, T) symmetric
    rc_lj: float = 2.5
    alpha: float = 0.4
    rc_r: float = 8.0
    kmax: int = 7
    k_e: float = 1.0
    dt: float = 0.002


def adjoint_mixture(ncell: int = 10, density: float = 0.8442, temperature: float = 1.0, seed: int = 5,
                    jitter: float = 0.05, rc_lj: float = 2.5, alpha: float = 0.4, rc_r: float = 8.0,
                    kmax: int = 7) -> AdjointSystem:
    """Two-species LJ + charge mixture: 4 ncell^3 atoms on an FCC lattice at
    rho* = 0.8442 (ncell = 10 gives N = 4000, L = 16.796), half A (q = +0.5),
    half B (q = -0.5) at random sites; eps_AA 1.0, eps_BB 0.5, eps_AB 0.75,
    sigma_AA 1.0, sigma_BB 0.88, sigma_AB 0.94 (Lorentz-Berthelot mean);
    Maxwell-Boltzmann velocities at T*; dt 0.002.  Ewald alpha 0.4 with a
    real-space cutoff of 8 sigma (erfc(3.2) = 6e-6) and k_max 7."""
    base = fcc_lattice(ncell, density, temperature, seed, jitter=jitter)
    n = base.n
    rng = np.random.default_rng(seed + 1000)
    typ = np.zeros(n, np.int32)
    typ[rng.permutation(n)[: n // 2]] = 1
    L = float(base.box[0])
    return AdjointSystem(box=L, pos=base.pos % L, vel=base.vel, type=typ, mass=np.ones(2), charge=np.array([0.5, -0.5]),
                         epsilon=np.array([[1.0, 0.75], [0.75, 0.5]]), sigma=np.array([[1.0, 0.94], [0.94, 0.88]]),
                         rc_lj=min(rc_lj, L / 2), alpha=alpha, rc_r=min(rc_r, L / 2), kmax=kmax)
