"""Generates the golden fixtures under tests/golden/ (run once, in a
container that has the reference sources; the fixtures are committed so the
GPU tests never need the reference at run time).

1. ewald_n100.json -- the reference's own Ewald known-answer case
   (benchmark/b2-ewald): 100 ions (type 0 q=-1, type 1 q=+1) in a 10^3
   periodic box, alpha = 1.112583061, real-space cutoff 4.9, kmax 30, with
   the published forces and total energy of benchmark/b2-ewald/espressopp/
   ewald_result.dat.  Positions and types come from
   benchmark/b2-ewald/caviar/ewald-n100.casl (`m1 add_atom aX at_position x y z`).

2. ref_*.npz -- outputs of the unmodified reference (oracle/_ref/ref_harness,
   compiled from the reference sources by oracle/Makefile) on small seeded
   systems: accelerations, canonical pair set, virial, kinetic energy, S(k),
   k-space and self energies, and a short trajectory.

3. nve_lj500.json, nve_ions500.json -- the reference's NVE energy record
   every 100 steps over 10^4 steps of a 500-atom LJ fluid (FCC 5^3 cells,
   rho* 0.8442, T* 0.72, rc 2.5, skin 0.3, dt 0.005) and of 500 ions (+-1,
   L = 16, LJ rc 2.5, Ewald alpha 0.6, real-space list radius 5.15, kmax 4,
   dt 0.005; the ions start from the reference's own state after 2000 steps,
   past the random start's relaxation, stored in the record): a hundred
   harness runs of 100 steps, each continuing from the
   previous run's final positions and velocities; total energy = the
   reference's kinetic energy + the potential energies the restatement
   evaluates at the reference's positions (the reference has no LJ energy
   and no list-consistent Ewald real-space energy).

4. writer_lj500/ -- the files the reference's `writer atom_data` writes for
   a 40-step run of that fluid (energy and temperature every 5 steps,
   pressure every 10, volume and xyz frames with ids, velocities and
   accelerations every 20; temperature_process and pressure_process on), with
   the script lines that declare the writer (WRITER_SCRIPT).

5. ref_langevin500.npz -- 20 steps of the reference's velocity_verlet_langevin
   (T 1.2, friction 0.5, kb 1) on that fluid: final positions, velocities
   and the kinetic-energy trace.

6. ref_berendsen500.npz, ref_nosehoover500.npz -- 30 velocity-Verlet steps
   of that fluid with the reference's `constraint berendsen` (T0 1.2,
   coupling 0.1, dt 0.005, every 2 steps) or `constraint nose_hoover` (type 1,
   T0 1.2, mass 20, kb 1, dt 0.005), temperature_process on.

7. ref_ewald_slab300.npz -- 300 ions (+-1) in a 10^3 box, LJ rc 2.5, Ewald
   alpha 0.8, k_max 4, list cutoff 4 (coef 1.03): the reference's forces with
   (a) z non-periodic, `slab_normal_axis z`, `slab_lz 30`, `epsilon_dipole 0`
   and (b) all periodic with `epsilon_dipole 1`, and (c) a 10-step run of (a).

8. ref_slab_correction300.npz -- the same ions with the reference's
   `force_field electrostatic_ewald_slab_correction` (lz 30, k_max 4) next to
   the slab Ewald sum: forces and a 10-step run with the normal axis z, and
   forces with the normal axis x.

9. ref_bench_lj4000.npz, ref_bench_ions8000.npz, ref_bench_lj1m.npz -- the
   unmodified reference on the benchmark systems themselves (the seeded
   generators of caviar_b200.workloads: 4000-atom LJ fluid, 8000 ions with
   Ewald alpha 0.3 / rc 10 / kmax 8, the 1,048,576-atom LJ fluid): the
   SHA-256 and size of its canonical pair set (checked here against the C
   restatement's, so the restatement is pinned at these sizes too),
   accelerations (every one for the two small systems, every 64th atom by
   id for the 1M system), virial, kinetic energy, S(k) and the k-space and
   self energies, and short trajectories (100 steps of the 4000-atom fluid,
   3 of the ions) under the reference's own rebuild trigger.  The LJ force
   states are the generators' lattices with sites displaced by up to 0.1
   (every force vanishes on the perfect lattice); the trajectories start
   from the benchmark states themselves.

10. ref_replicas.npz -- the unmodified reference on twelve replicas of the
   batch workload (64 ... 2048 atoms, every size class boundary), each run as
   its own system with neighbour-list radius = ghost cutoff = L/2
   (cutoff_extra_coef 1, the largest its one-ghost-image scheme allows; its
   Ewald real-space sum then covers the minimum-image pairs within L/2):
   accelerations, virial, kinetic energy, k-space and self energies.

11. ref_ljjump500.npz -- the reference's forces and virial with `f_lj
   jump_tol 0.9` on a 500-atom fluid in which twenty atoms were moved to
   0.85-0.93 sigma from their nearest neighbour (jump_system()).

12. ref_allatom300.npz -- the reference with `neigh all_atom_test` on 300
   ions (all_atom_system()): forces, virial, S(k), k-space energy, the
   SHA-256 and size of its pair set (every owned pair and every ghost image)
   and a 10-step run.

Usage:  python tests/golden/make_golden.py [/path/to/reference]
        [--bench-only | --replicas-only | --nve-only | --jump-only]
The reference root defaults to $CAVIAR_REFERENCE_ROOT, else to a directory
named `reference` beside this repository.
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from caviar_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def ewald_n100(ref_root: str) -> dict:
    casl = os.path.join(ref_root, "benchmark", "b2-ewald", "caviar", "ewald-n100.casl")
    dat = os.path.join(ref_root, "benchmark", "b2-ewald", "espressopp", "ewald_result.dat")
    pos, typ = [], []
    pat = re.compile(r"^\s*m1\s+add_atom\s+a([12])\s+at_position\s+(\S+)\s+(\S+)\s+(\S+)")
    with open(casl) as f:
        for line in f:
            m = pat.match(line)
            if m:
                typ.append(int(m.group(1)) - 1)
                pos.append([float(m.group(2)), float(m.group(3)), float(m.group(4))])
    forces, energy = [], None
    with open(dat) as f:
        lines = f.read().splitlines()
    for k, line in enumerate(lines):
        if line.strip().startswith("total_energy"):
            energy = float(lines[k + 1])
        m = re.match(r"^\s*\{\s*(\S+)\s+(\S+)\s+(\S+)\s*\}", line)
        if m:
            forces.append([float(m.group(1)), float(m.group(2)), float(m.group(3))])
    assert len(pos) == 100 and len(forces) == 100 and energy is not None
    return {
        "source": "benchmark/b2-ewald (caviar/ewald-n100.casl positions, espressopp/ewald_result.dat forces)",
        "box": [0.0, 10.0], "alpha": 1.112583061, "rcut": 4.9, "kmax": 30,
        "charge_by_type": [-1.0, 1.0], "mass_by_type": [1.0, 1.0],
        "type": typ, "pos": pos, "force": forces, "total_energy": energy,
    }


def small_systems():
    out = {}
    # plain LJ, FCC 5^3 cells (500 atoms, L = 8.40 >= 2 rl), lattice jittered by 0.1
    out["lj500"] = W.fcc_lattice(5, 0.8442, 0.72, seed=11, jitter=0.1)
    # two-type LJ mixture with cutoff_list and Lorentz-Berthelot-like sigma
    s = W.fcc_lattice(5, 0.8442, 1.0, seed=12, jitter=0.1)
    s.type = (np.arange(s.n) % 3 == 0).astype(np.int32)
    s.mass = np.array([1.0, 2.0])
    s.charge = np.zeros(2)
    s.lj = W.LJParams(cutoff=2.5, epsilon=np.array([[1.0, 0.75], [0.75, 0.5]]),
                      sigma=np.array([[1.0, 0.94], [0.94, 0.88]]),
                      cutoff_list=np.array([[2.5, 2.2], [2.2, 2.0]]))
    s.name = "ljmix500"
    out["ljmix500"] = s
    # charged LJ + Ewald r + k (L = 16, rl = 5.15, kmax 4)
    out["ions500"] = W.random_ions(500, 16.0, seed=13, rc=5.0, kmax=4, alpha=0.6)
    return out


def save_ref(name, s, nsteps=20):
    f = O.run_reference(s, "forces")
    r = O.run_reference(s, "run", nsteps=nsteps)
    d = dict(
        lo=s.lo, hi=s.hi, mass=s.mass, charge=s.charge, pos=s.pos, vel=s.vel, type=s.type,
        cutoff=s.cutoff, coef=s.coef, ghost_cutoff=s.ghost_cutoff, dt=s.dt,
        lj_cutoff=s.lj.cutoff if s.lj else -1.0,
        lj_eps=s.lj.epsilon if s.lj else np.zeros((1, 1)),
        lj_sigma=s.lj.sigma if s.lj else np.zeros((1, 1)),
        lj_cutoff_list=s.lj.cutoff_list if (s.lj is not None and s.lj.cutoff_list is not None) else np.zeros((0, 0)),
        ewr_alpha=s.ewald_r.alpha if s.ewald_r else -1.0,
        ewk_alpha=s.ewald_k.alpha if s.ewald_k else -1.0,
        ewk_kmax=np.array(s.ewald_k.kmax if s.ewald_k else (0, 0, 0)),
        ref_acc=f["acc"], ref_pairs=f["pairs"], ref_virial=f["virial"], ref_ke=f["ke"],
        ref_sk=f.get("sk", np.zeros(0)), ref_ek=f.get("ek_kspace", 0.0), ref_eself=f.get("ek_self", 0.0),
        run_steps=nsteps, run_pos=r["pos"], run_vel=r["vel"], run_acc=r["acc"], run_ke=r["ke_trace"],
        run_virial=r["vir_trace"],
    )
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **d)


def nve_trace(s, nblocks: int = 100, block: int = 100) -> list:
    """Total energy of the reference's own NVE run every `block` steps:
    `nblocks` harness runs of `block` steps, each continuing from the previous
    run's final positions and velocities (a restart recomputes the forces of
    those positions, as the continuing run has them); the energy of each
    state is the reference's kinetic energy plus the potential energies the
    restatement evaluates there (LJ of the reference's linear force-shifted
    potential, Ewald real space over the list pairs, k space, self)."""
    cur = s.copy()
    e = []
    o = O.Oracle(cur, policy=O.POLICY_REFERENCE)
    for b in range(nblocks + 1):
        o.set_atoms(cur.pos, cur.vel, cur.type)
        o.setup()  # list and forces of this state (the k-space energy uses its S(k))
        sc = o.energy()
        e.append(sc["ke"] + sc["e_lj"] + sc["e_ewald_r"] + sc["e_ewald_k"] + sc["e_self"])
        if b == nblocks:
            break
        r = O.run_reference(cur, "run", block)
        order = np.argsort(r["id"].astype(np.int64))
        cur = cur.copy()
        cur.pos = r["pos"].reshape(-1, 3)[order]
        cur.vel = r["vel"].reshape(-1, 3)[order]
    return e


NVE_SYSTEMS = {
    "lj500": ("fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)",
              lambda: W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)),
    "ions500": ("random_ions(500, 16.0, seed=13, rc=5.0, kmax=4, alpha=0.6)",
                lambda: W.random_ions(500, 16.0, seed=13, rc=5.0, kmax=4, alpha=0.6)),
}


def nve(name: str, nblocks: int = 100, block: int = 100, equilibrate: int = 0) -> dict:
    """The trace of NVE_SYSTEMS[name]; with equilibrate > 0 the trace starts
    from the reference's own state after that many steps (past the start's
    relaxation transient) and the record holds that state."""
    desc, make = NVE_SYSTEMS[name]
    s = make()
    out = {"system": desc, "steps_per_record": block, "n": s.n, "equilibrate_steps": equilibrate}
    if equilibrate:
        r = O.run_reference(s, "run", equilibrate)
        order = np.argsort(r["id"].astype(np.int64))
        s.pos = r["pos"].reshape(-1, 3)[order]
        s.vel = r["vel"].reshape(-1, 3)[order]
        out["pos0"] = s.pos.tolist()
        out["vel0"] = s.vel.tolist()
    out["total_energy"] = nve_trace(s, nblocks, block)
    return out


NVE_EQUILIBRATE = {"lj500": 0, "ions500": 2000}


WRITER_SCRIPT = """writer atom_data w
w set_atom_data adata
w set_domain dom
w energy_step 5
w temperature_step 5
w pressure_step 10
w volume_step 20
w xyz_step 20
w xyz_output_id 1
w xyz_output_velocity 1
w xyz_output_acceleration 1
adata temperature_process 1
adata pressure_process 1
sim add_writer w
"""
WRITER_FILES = ("o_energy.txt", "o_temperature.txt", "o_pressure.txt", "o_volume.txt", "o_xyz.xyz")


def writer_lj500(nsteps: int = 40) -> None:
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    r = O.run_reference(s, "run", nsteps, extra=WRITER_SCRIPT, collect=WRITER_FILES)
    out = os.path.join(HERE, "writer_lj500")
    os.makedirs(out, exist_ok=True)
    for name in WRITER_FILES:
        with open(os.path.join(out, name), "w") as f:
            f.write(r["files"][name])
    with open(os.path.join(out, "script_extra.casl"), "w") as f:
        f.write(WRITER_SCRIPT)


LANGEVIN_SCRIPT = """sim integrator_type velocity_verlet_langevin
sim temperature 1.2
sim friction 0.5
sim kb 1.0
"""


def langevin500(nsteps: int = 20) -> None:
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    r = O.run_reference(s, "run", nsteps, extra=LANGEVIN_SCRIPT)
    order = np.argsort(r["id"].astype(np.int64))
    np.savez_compressed(os.path.join(HERE, "ref_langevin500.npz"), pos=r["pos"].reshape(-1, 3)[order],
                        vel=r["vel"].reshape(-1, 3)[order], ke=r["ke_trace"], nsteps=nsteps, script=LANGEVIN_SCRIPT)


THERMOSTAT_SCRIPTS = {
    "berendsen500": """constraint berendsen c1
c1 set_atom_data adata
c1 temperature 1.2
c1 coupling 0.1
c1 dt 0.005
c1 step 2
adata temperature_process 1
sim add_constraint c1
""",
    "nosehoover500": """constraint nose_hoover c1
c1 set_atom_data adata
c1 temperature 1.2
c1 type 1
c1 mass 20.0
c1 kb 1.0
c1 dt 0.005
adata temperature_process 1
sim add_constraint c1
""",
}


def thermostats(nsteps: int = 30) -> None:
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    for name, extra in THERMOSTAT_SCRIPTS.items():
        r = O.run_reference(s, "run", nsteps, extra=extra)
        order = np.argsort(r["id"].astype(np.int64))
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), pos=r["pos"].reshape(-1, 3)[order],
                            vel=r["vel"].reshape(-1, 3)[order], acc=r["acc"].reshape(-1, 3)[order],
                            ke=r["ke_trace"], nsteps=nsteps, script=extra)


SLAB_SCRIPTS = {
    "slab": "f_ek slab_normal_axis z\nf_ek slab_lz 30.0\nf_ek epsilon_dipole 0.0\n",
    "dipole": "f_ek epsilon_dipole 1.0\n",
}


def slab_system(periodic_z: bool):
    s = W.random_ions(300, 10.0, 21, rc=4.0, coef=1.03, kmax=4, alpha=0.8)
    s.bc = (1, 1, 1 if periodic_z else 0)
    return s


def ewald_slab() -> None:
    out = {}
    for name, extra in SLAB_SCRIPTS.items():
        s = slab_system(name != "slab")
        r = O.run_reference(s, "forces", extra=extra)
        order = np.argsort(r["id"].astype(np.int64))
        out[f"{name}_acc"] = r["acc"].reshape(-1, 3)[order]
        out[f"{name}_script"] = extra
    s = slab_system(False)
    r = O.run_reference(s, "run", 10, extra=SLAB_SCRIPTS["slab"])
    order = np.argsort(r["id"].astype(np.int64))
    out["slab_run_pos"] = r["pos"].reshape(-1, 3)[order]
    out["slab_run_vel"] = r["vel"].reshape(-1, 3)[order]
    np.savez_compressed(os.path.join(HERE, "ref_ewald_slab300.npz"), **out)


def slab_correction() -> None:
    out = {}
    for ax, name in ((2, "z"), (0, "x")):
        s = W.random_ions(300, 10.0, 21, rc=4.0, coef=1.03, kmax=4, alpha=0.8)
        s.bc = (0, 1, 1) if ax == 0 else (1, 1, 0)
        extra = (f"f_ek slab_normal_axis {name}\nf_ek slab_lz 30.0\n"
                 "force_field electrostatic_ewald_slab_correction f_sc\nf_sc set_atom_data adata\n"
                 f"f_sc set_domain dom\nf_sc slab_normal_axis {name}\nf_sc lz 30.0\nf_sc k_max 4\n"
                 "sim add_force_field f_sc\n")
        r = O.run_reference(s, "forces", extra=extra)
        order = np.argsort(r["id"].astype(np.int64))
        out[f"{name}_acc"] = r["acc"].reshape(-1, 3)[order]
        out[f"{name}_script"] = extra
        if name == "z":
            r = O.run_reference(s, "run", 10, extra=extra)
            order = np.argsort(r["id"].astype(np.int64))
            out["z_run_pos"] = r["pos"].reshape(-1, 3)[order]
            out["z_run_vel"] = r["vel"].reshape(-1, 3)[order]
    np.savez_compressed(os.path.join(HERE, "ref_slab_correction300.npz"), **out)


def random_velocity500(seed: int = 7, amplitude: float = 1.5) -> None:
    """Atom_data::add_random_velocity of the unmodified reference on a
    two-species system with different masses (the centre-of-mass correction
    is mass-weighted): its velocities, for the CASL front end's keyword."""
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=9, jitter=0.05)
    rng = np.random.default_rng(9)
    s.type = (rng.random(s.n) < 0.4).astype(np.int32)
    s.mass = np.array([1.0, 2.5])
    s.charge = np.zeros(2)
    s.lj = W.LJParams(cutoff=2.5, epsilon=np.ones((2, 2)), sigma=np.ones((2, 2)))
    r = O.run_reference(s, "randvel", mode_args=(seed, amplitude))
    order = np.argsort(r["id"].astype(np.int64))
    np.savez_compressed(os.path.join(HERE, "ref_randvel500.npz"), pos=s.pos, type=s.type, mass=s.mass,
                        box=s.box, seed=seed, amplitude=amplitude, vel=r["vel"].reshape(-1, 3)[order])


# replica sizes of the batch tests: every size class and class boundary
REPLICA_SIZES = [64, 100, 257, 511, 512, 513, 777, 1024, 1025, 1500, 2047, 2048]


def replicas() -> None:
    """The unmodified reference on each replica of replica_batch(sizes=
    REPLICA_SIZES, seed=5), run as its own system (workloads.replica_system:
    list radius = ghost cutoff = L/2, cutoff_extra_coef 1): accelerations in
    id order, virial, kinetic energy, k-space and self energies."""
    b = W.replica_batch(sizes=REPLICA_SIZES, seed=5)
    out = {"sizes": np.asarray(REPLICA_SIZES), "seed": 5}
    acc, vir, ke, ek, es = [], [], [], [], []
    for r in range(len(REPLICA_SIZES)):
        s = W.replica_system(b, r)
        f = O.run_reference(s, "forces")
        order = np.argsort(f["id"].astype(np.int64))
        acc.append(f["acc"].reshape(-1, 3)[order])
        vir.append(float(f["virial"]))
        ke.append(float(f["ke"]))
        ek.append(float(f["ek_kspace"]))
        es.append(float(f["ek_self"]))
    out.update(acc=np.concatenate(acc), virial=np.asarray(vir), ke=np.asarray(ke), e_k=np.asarray(ek),
               e_self=np.asarray(es))
    np.savez_compressed(os.path.join(HERE, "ref_replicas.npz"), **out)


def jump_system():
    """500-atom LJ fluid with twenty atoms moved towards their nearest
    neighbour (to 0.85-0.93 sigma) and the reference's lj jump_tol 0.9
    (pairs closer than sqrt(0.9) get the coefficient of r^2 = 0.9)."""
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=17, jitter=0.05)
    rng = np.random.default_rng(17)
    L = float(s.box[0])
    pos = s.pos.copy()
    for i in rng.choice(s.n, size=20, replace=False):
        d = pos - pos[i]
        d -= L * np.round(d / L)
        r = np.linalg.norm(d, axis=1)
        r[i] = np.inf
        j = int(np.argmin(r))
        target = rng.uniform(0.85, 0.93)
        pos[i] = pos[i] + d[j] / r[j] * (r[j] - target)
    s.pos = pos % L
    s.lj.jump_tol = 0.9
    return s


def jump500() -> None:
    s = jump_system()
    f = O.run_reference(s, "forces")
    order = np.argsort(f["id"].astype(np.int64))
    np.savez_compressed(os.path.join(HERE, "ref_ljjump500.npz"), pos=s.pos, acc=f["acc"].reshape(-1, 3)[order],
                        virial=f["virial"], jump_tol=s.lj.jump_tol)


def all_atom_system():
    """300 ions (+-1) in a 10^3 box, LJ rc 2.5, Ewald alpha 0.8, k_max 3,
    list radius 3.09 (ghost cutoff the same)."""
    return W.random_ions(300, 10.0, seed=23, rc=3.0, coef=1.03, kmax=3, alpha=0.8)


def all_atom300(nsteps: int = 10) -> None:
    """The reference with `neigh all_atom_test`: forces, virial, its pair
    set (every owned pair and ghost image) and a 10-step run."""
    s = all_atom_system()
    extra = "neigh all_atom_test\n"
    f = O.run_reference(s, "forces", extra=extra)
    order = np.argsort(f["id"].astype(np.int64))
    r = O.run_reference(s, "run", nsteps=nsteps, extra=extra)
    orr = np.argsort(r["id"].astype(np.int64))
    np.savez_compressed(os.path.join(HERE, "ref_allatom300.npz"), acc=f["acc"].reshape(-1, 3)[order],
                        virial=f["virial"], pairs_sha256=pair_digest(f["pairs"].reshape(-1, 5)),
                        npairs=f["pairs"].size // 5, sk=f["sk"], ek=f["ek_kspace"],
                        run_steps=nsteps, run_pos=r["pos"].reshape(-1, 3)[orr], run_vel=r["vel"].reshape(-1, 3)[orr])


def pair_digest(pairs: np.ndarray) -> str:
    """SHA-256 of a canonical pair set (n x 5 int32, little endian, row major)."""
    return hashlib.sha256(np.ascontiguousarray(pairs, dtype="<i4").tobytes()).hexdigest()


BENCH_SYSTEMS = {
    # name: (generator, keyword arguments of the force state, trajectory steps,
    #        stride of the stored accelerations).  The LJ force states displace
    #        the lattice sites by up to 0.1 (on the perfect lattice every force
    #        vanishes); trajectories start from the benchmark state itself.
    "lj4000": (W.config_lj_4000, {"jitter": 0.1}, 100, 1),
    "ions8000": (W.config_ions_8000, {}, 3, 1),
    "lj1m": (W.config_lj_1m, {"jitter": 0.1}, 0, 64),
}


def bench_systems() -> None:
    for name, (gen, kw, nsteps, stride) in BENCH_SYSTEMS.items():
        s = gen(**kw)
        f = O.run_reference(s, "forces")
        order = np.argsort(f["id"].astype(np.int64))
        acc = f["acc"].reshape(-1, 3)[order]
        pairs = f["pairs"].reshape(-1, 5)
        o = O.Oracle(s)
        o.setup()
        opairs = o.pairs()
        assert np.array_equal(opairs, pairs), f"{name}: restatement pair set differs from the reference's"
        del opairs
        d = dict(generator=gen.__name__, generator_kwargs=json.dumps(kw), n=s.n, pairs_sha256=pair_digest(pairs),
                 npairs=pairs.shape[0],
                 acc_stride=stride, ref_acc=acc[::stride], ref_virial=f["virial"], ref_ke=f["ke"],
                 ref_sk=f.get("sk", np.zeros(0)), ref_ek=f.get("ek_kspace", 0.0), ref_eself=f.get("ek_self", 0.0),
                 run_steps=nsteps)
        if nsteps:
            r = O.run_reference(gen(), "run", nsteps=nsteps)
            order = np.argsort(r["id"].astype(np.int64))
            d.update(run_pos=r["pos"].reshape(-1, 3)[order], run_vel=r["vel"].reshape(-1, 3)[order],
                     run_ke=r["ke_trace"])
        np.savez_compressed(os.path.join(HERE, f"ref_bench_{name}.npz"), **d)
        print(name, "pairs", pairs.shape[0], "ok")


def reference_root() -> str:
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if args:
        return args[0]
    return os.environ.get("CAVIAR_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))


def main():
    ref_root = reference_root()
    if "--bench-only" in sys.argv:
        O.build(ref_root)
        bench_systems()
        return
    if "--nve-only" in sys.argv:
        O.build(ref_root)
        for name in NVE_SYSTEMS:
            with open(os.path.join(HERE, f"nve_{name}.json"), "w") as f:
                json.dump(nve(name, equilibrate=NVE_EQUILIBRATE[name]), f)
        return
    if "--jump-only" in sys.argv:
        O.build(ref_root)
        jump500()
        all_atom300()
        return
    if "--replicas-only" in sys.argv:
        O.build(ref_root)
        replicas()
        return
    g = ewald_n100(ref_root)
    with open(os.path.join(HERE, "ewald_n100.json"), "w") as f:
        json.dump(g, f, indent=0)
    O.build(ref_root)
    for name, s in small_systems().items():
        save_ref(name, s)
    for name in NVE_SYSTEMS:
        with open(os.path.join(HERE, f"nve_{name}.json"), "w") as f:
            json.dump(nve(name, equilibrate=NVE_EQUILIBRATE[name]), f)
    writer_lj500()
    langevin500()
    thermostats()
    ewald_slab()
    slab_correction()
    random_velocity500()
    bench_systems()
    replicas()
    jump500()
    all_atom300()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
