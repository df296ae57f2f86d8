"""Python access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

* `Oracle` -- ctypes binding of the FP64 C restatement (oracle.c, built into
  oracle/_build/liboracle.so by oracle/Makefile).
* `run_reference` -- runs the unmodified reference compiled from its own
  sources (oracle/_ref/ref_harness) on an `MDSystem`: writes the CASL script
  with the reference's own keywords and a binary state file, runs the
  harness, reads back its FP64 output.

Only tests/, __graft_entry__.smoke and bench.py's CPU-baseline leg use this
module; the product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
import time
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
HARNESS_PATH = os.path.join(HERE, "_ref", "ref_harness")
# the reference with the B200 integration layer (`md_simulator b200` / `b200_fp64`)
HARNESS_B200_PATH = os.path.join(HERE, "_ref", "ref_harness_b200")

POLICY_DISPLACEMENT = 0
POLICY_REFERENCE = 1
POLICY_EVERY_STEP = 2

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lib = None


def build(reference_root: Optional[str] = None, quiet: bool = True) -> None:
    """Compile the restatement (and, when the reference sources are present,
    the reference harness, and the reference with the B200 integration layer
    when libcaviar_b200.so is built) with oracle/Makefile."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE], check=True, stdout=out)
    if reference_root and os.path.isdir(reference_root):
        subprocess.run(["make", "-C", HERE, "-j8", "ref", f"REF={reference_root}"], check=True, stdout=out)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "caviar_b200", "libcaviar_b200.so")):
            subprocess.run(["make", "-C", HERE, "ref_b200", f"REF={reference_root}"], check=True, stdout=out)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [_dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, _dp, _dp]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_atoms.argtypes = [ctypes.c_void_p, ctypes.c_int64, _dp, _dp, _ip, _ip]
        L.orc_set_neighborlist.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int]
        L.orc_set_lj.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, ctypes.c_int, ctypes.c_double]
        L.orc_set_ewald_r.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_double]
        L.orc_set_ewald_k.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double]
        L.orc_set_integrator.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        for f in ("orc_setup", "orc_step", "orc_build_list", "orc_compute_forces", "orc_energy"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.orc_pairs.restype = ctypes.c_int64
        L.orc_pairs.argtypes = [ctypes.c_void_p, _ip]
        L.orc_get_state.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_n_kvec_used.restype = ctypes.c_int64
        L.orc_n_kvec_used.argtypes = [ctypes.c_void_p]
        L.orc_get_sk.argtypes = [ctypes.c_void_p, _dp]
        L.orc_get_scalars.argtypes = [ctypes.c_void_p, _dp]
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


class Oracle:
    """The FP64 restatement for one periodic system."""

    def __init__(self, system, policy: int = POLICY_DISPLACEMENT, all_atom_test: bool = False):
        L = lib()
        self._keep = []
        s = system
        lo = np.ascontiguousarray(s.lo, np.float64)
        hi = np.ascontiguousarray(s.hi, np.float64)
        bc = (ctypes.c_int * 3)(*[int(b) for b in s.bc])
        mass = np.ascontiguousarray(s.mass, np.float64)
        charge = np.ascontiguousarray(s.charge, np.float64)
        self.h = L.orc_create(_d(lo), _d(hi), bc, s.n_types, _d(mass), _d(charge))
        self.n = s.n
        self.set_atoms(s.pos, s.vel, s.type, s.mol)
        L.orc_set_neighborlist(self.h, s.cutoff, s.coef, s.ghost_cutoff, int(all_atom_test))
        if s.lj is not None:
            eps = np.ascontiguousarray(s.lj.epsilon, np.float64)
            sig = np.ascontiguousarray(s.lj.sigma, np.float64)
            cl = None if s.lj.cutoff_list is None else np.ascontiguousarray(s.lj.cutoff_list, np.float64)
            L.orc_set_lj(self.h, s.lj.cutoff, _d(eps), _d(sig), _d(cl), int(s.lj.ignore_intra_molecule),
                         float(s.lj.jump_tol))
        if s.ewald_r is not None:
            lam = None if s.ewald_r.lam is None else np.ascontiguousarray(s.ewald_r.lam, np.float64)
            L.orc_set_ewald_r(self.h, s.ewald_r.alpha, s.ewald_r.k_electrostatic, _d(lam), s.ewald_r.cutoff)
        if s.ewald_k is not None:
            kx, ky, kz = s.ewald_k.kmax
            L.orc_set_ewald_k(self.h, s.ewald_k.alpha, kx, ky, kz, s.ewald_k.k_electrostatic)
        L.orc_set_integrator(self.h, s.dt, s.k_b, policy)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_atoms(self, pos, vel, typ, mol=None):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        typ = np.ascontiguousarray(typ, np.int32)
        molp = None
        if mol is not None:
            mol = np.ascontiguousarray(mol, np.int32)
            molp = mol.ctypes.data_as(_ip)
        self.n = pos.shape[0]
        rc = lib().orc_set_atoms(self.h, self.n, _d(pos), _d(vel), typ.ctypes.data_as(_ip), molp)
        if rc != 0:
            raise ValueError("atom type out of range")

    def setup(self):
        lib().orc_setup(self.h)

    def build_list(self):
        lib().orc_build_list(self.h)

    def compute_forces(self):
        lib().orc_compute_forces(self.h)

    def step(self, nsteps: int = 1):
        for _ in range(nsteps):
            if lib().orc_step(self.h) != 0:
                raise FloatingPointError("NaN acceleration")

    def pairs(self) -> np.ndarray:
        m = lib().orc_pairs(self.h, None)
        out = np.zeros((m, 5), np.int32)
        lib().orc_pairs(self.h, out.ctypes.data_as(_ip))
        return out

    def state(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        acc = np.zeros((self.n, 3))
        lib().orc_get_state(self.h, _d(pos), _d(vel), _d(acc))
        return pos, vel, acc

    def sk(self) -> np.ndarray:
        m = lib().orc_n_kvec_used(self.h)
        out = np.zeros((m, 2))
        lib().orc_get_sk(self.h, _d(out))
        return out[:, 0] + 1j * out[:, 1]

    def energy(self) -> Dict[str, float]:
        lib().orc_energy(self.h)
        return self.scalars()

    def scalars(self) -> Dict[str, float]:
        out = np.zeros(9)
        lib().orc_get_scalars(self.h, _d(out))
        keys = ["virial", "ke", "e_lj", "e_ewald_r", "e_ewald_k", "e_self", "n_builds", "n_ghost", "dof"]
        return dict(zip(keys, out.tolist()))


def replica_forces(n, pos, typ, L, mass, charge, eps, sigma, rc_lj, alpha, rc_r, kmax, k_e=1.0):
    """FP64 minimum-image forces of one small replica; returns (acc, energies)."""
    Lb = lib()
    f = Lb.orc_replica_forces
    f.argtypes = [ctypes.c_int64, _dp, _ip, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp, _dp]
    f.restype = None
    pos = np.ascontiguousarray(pos, np.float64)
    typ = np.ascontiguousarray(typ, np.int32)
    acc = np.zeros((n, 3))
    en = np.zeros(5)
    arrs = [np.ascontiguousarray(x, np.float64) for x in (mass, charge, eps, sigma)]
    f(n, _d(pos), typ.ctypes.data_as(_ip), L, len(arrs[0]), *[_d(a) for a in arrs], rc_lj, alpha, rc_r, kmax, k_e,
      _d(acc), _d(en))
    return acc, dict(zip(["e_lj", "e_ewald_r", "e_ewald_k", "e_self", "virial"], en.tolist()))


def replica_run(n, pos, vel, typ, L, mass, charge, eps, sigma, rc_lj, alpha, rc_r, kmax, k_e, dt, nsteps):
    """FP64 velocity-Verlet run of one small replica; returns (pos, vel, acc)."""
    Lb = lib()
    f = Lb.orc_replica_run
    f.argtypes = [ctypes.c_int64, _dp, _dp, _dp, _ip, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp,
                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                  ctypes.c_int64]
    f.restype = None
    p = np.array(pos, np.float64)
    v = np.array(vel, np.float64)
    a = np.zeros((n, 3))
    typ = np.ascontiguousarray(typ, np.int32)
    arrs = [np.ascontiguousarray(x, np.float64) for x in (mass, charge, eps, sigma)]
    f(n, _d(p), _d(v), _d(a), typ.ctypes.data_as(_ip), L, len(arrs[0]), *[_d(x) for x in arrs], rc_lj, alpha, rc_r,
      kmax, k_e, dt, nsteps)
    return p, v, a


class AdjOracle:
    """FP64 trajectory adjoint restatement (adjoint.c) for one periodic cube."""

    def __init__(self, sysd):
        """sysd: caviar_b200.workloads.AdjointSystem (or anything with its fields)."""
        L = lib()
        vp = ctypes.c_void_p
        L.orc_adj_create.restype = vp
        L.orc_adj_create.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, _ip]
        L.orc_adj_destroy.argtypes = [vp]
        L.orc_adj_set_params.argtypes = [vp, _dp, _dp, _dp]
        L.orc_adj_forces.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_adj_force_vjp.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_adj_loss.restype = ctypes.c_double
        L.orc_adj_loss.argtypes = [vp, _dp, _dp, ctypes.c_int64, _dp, _dp]
        L.orc_adj_loss_grad.restype = ctypes.c_double
        L.orc_adj_loss_grad.argtypes = [vp, _dp, _dp, ctypes.c_int64, ctypes.c_int64, _dp, _dp, _dp, _dp, _dp]
        self.L = L
        self.s = sysd
        self.n = int(sysd.pos.shape[0])
        self.nt = len(sysd.mass)
        self._typ = np.ascontiguousarray(sysd.type, np.int32)
        a = [np.ascontiguousarray(x, np.float64) for x in (sysd.mass, sysd.charge, sysd.epsilon, sysd.sigma)]
        self.h = L.orc_adj_create(self.n, float(sysd.box), self.nt, *[_d(x) for x in a], sysd.rc_lj, sysd.alpha,
                                  sysd.rc_r, sysd.kmax, sysd.k_e, sysd.dt, self._typ.ctypes.data_as(_ip))
        if not self.h:
            raise ValueError("orc_adj_create rejected the system")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_adj_destroy(self.h)
            self.h = None

    def set_params(self, eps=None, sigma=None, charge=None):
        arr = [None if x is None else np.ascontiguousarray(x, np.float64) for x in (eps, sigma, charge)]
        self.L.orc_adj_set_params(self.h, *[None if x is None else _d(x) for x in arr])

    def forces(self, pos):
        pos = np.ascontiguousarray(pos, np.float64)
        nt = self.nt
        f, e = np.zeros((self.n, 3)), np.zeros(4)
        ge, gs, gq = np.zeros((nt, nt)), np.zeros((nt, nt)), np.zeros(nt)
        self.L.orc_adj_forces(self.h, _d(pos), _d(f), _d(e), _d(ge), _d(gs), _d(gq))
        return f, e, {"eps": ge, "sigma": gs, "charge": gq}

    def force_vjp(self, pos, u):
        pos = np.ascontiguousarray(pos, np.float64)
        u = np.ascontiguousarray(u, np.float64)
        nt = self.nt
        w = np.zeros((self.n, 3))
        ge, gs, gq = np.zeros((nt, nt)), np.zeros((nt, nt)), np.zeros(nt)
        self.L.orc_adj_force_vjp(self.h, _d(pos), _d(u), _d(w), _d(ge), _d(gs), _d(gq))
        return w, {"eps": ge, "sigma": gs, "charge": gq}

    def loss(self, pos0, vel0, M):
        p = np.ascontiguousarray(pos0, np.float64)
        v = np.ascontiguousarray(vel0, np.float64)
        return self.L.orc_adj_loss(self.h, _d(p), _d(v), M, None, None)

    def loss_grad(self, pos0, vel0, M, K):
        p = np.ascontiguousarray(pos0, np.float64)
        v = np.ascontiguousarray(vel0, np.float64)
        nt = self.nt
        gp, gv = np.zeros((self.n, 3)), np.zeros((self.n, 3))
        ge, gs, gq = np.zeros((nt, nt)), np.zeros((nt, nt)), np.zeros(nt)
        J = self.L.orc_adj_loss_grad(self.h, _d(p), _d(v), M, K, _d(gp), _d(gv), _d(ge), _d(gs), _d(gq))
        return J, {"pos": gp, "vel": gv, "eps": ge, "sigma": gs, "charge": gq}


# --------------------------------------------------------------- reference


def casl_script(system, nsteps: int = 1, rebuild_test: bool = False, extra: str = "",
                simulator: str = "basic") -> str:
    """The CASL objects of the hot path, with the reference's own keywords
    (domain.cpp:206-266, atom_data.cpp:78-306, neighborlist.cpp:193-251,
    lj.cpp:42-147, electrostatic_ewald_r.cpp:38-88, electrostatic_ewald_k.cpp:48-143,
    md_simulator.cpp:58-233).  Atoms are added by the harness, not here."""
    s = system
    r = repr
    lines = ["domain box dom"]
    for ax, a in zip("xyz", range(3)):
        lines.append(f"dom {ax}min {r(float(s.lo[a]))} {ax}max {r(float(s.hi[a]))}")
    lines.append("dom boundary_condition " + " ".join(str(int(b)) for b in s.bc))
    lines.append("dom generate")
    lines += ["atom_data basic adata", f"adata ghost_cutoff {r(float(s.ghost_cutoff))}", f"adata k_b {r(float(s.k_b))}",
              "adata set_domain dom"]
    for t in range(s.n_types):
        lines.append(f"adata add_type_mass {t} {r(float(s.mass[t]))}")
        lines.append(f"adata add_type_charge {t} {r(float(s.charge[t]))}")
    lines += ["neighborlist basic neigh", "neigh set_atom_data adata", "neigh set_domain dom",
              f"neigh cutoff {r(float(s.cutoff))}", f"neigh cutoff_extra_coef {r(float(s.coef))}",
              "neigh make_verlet_list_from_cell_list"]
    if rebuild_test:
        lines.append("neigh rebuild_test")
    ffs = []
    if s.lj is not None:
        ffs.append("f_lj")
        lines += ["force_field lj f_lj", f"f_lj cutoff {r(float(s.lj.cutoff))}"]
        T = s.n_types
        for i in range(T):
            for j in range(T):
                lines.append(f"f_lj epsilon {i} {j} {r(float(s.lj.epsilon[i][j]))}")
                lines.append(f"f_lj sigma {i} {j} {r(float(s.lj.sigma[i][j]))}")
                if s.lj.cutoff_list is not None:
                    lines.append(f"f_lj cutoff_list {i} {j} {r(float(s.lj.cutoff_list[i][j]))}")
        if getattr(s.lj, "jump_tol", 0.0) > 0:
            lines.append(f"f_lj jump_tol {r(float(s.lj.jump_tol))}")
        lines += ["f_lj set_neighborlist neigh", "f_lj set_atom_data adata", "f_lj set_domain dom"]
    if s.ewald_r is not None:
        ffs.append("f_er")
        cut = s.ewald_r.cutoff if s.ewald_r.cutoff > 0 else s.cutoff
        lines += ["force_field electrostatic_ewald_r f_er", f"f_er alpha {r(float(s.ewald_r.alpha))}",
                  f"f_er k_electrostatic {r(float(s.ewald_r.k_electrostatic))}", f"f_er cutoff {r(float(cut))}",
                  "f_er set_neighborlist neigh", "f_er set_atom_data adata"]
    if s.ewald_k is not None:
        ffs.append("f_ek")
        kx, ky, kz = s.ewald_k.kmax
        lines += ["force_field electrostatic_ewald_k f_ek", f"f_ek alpha {r(float(s.ewald_k.alpha))}",
                  f"f_ek kx_max {kx}", f"f_ek ky_max {ky}", f"f_ek kz_max {kz}",
                  f"f_ek k_electrostatic {r(float(s.ewald_k.k_electrostatic))}",
                  "f_ek set_atom_data adata", "f_ek set_domain dom"]
    lines += [f"md_simulator {simulator} sim", "sim set_atom_data adata", "sim integrator_type velocity_verlet"]
    for f in ffs:
        lines.append(f"sim add_force_field {f}")
    lines += ["sim add_neighborlist neigh", "sim initial_step 0", f"sim final_step {max(1, nsteps)}",
              f"sim dt {r(float(s.dt))}"]
    return "\n".join(lines) + "\n" + extra


def write_state(path: str, system) -> None:
    n = system.n
    rec = np.zeros(n, dtype=[("type", "<i4"), ("mol", "<i4"), ("pos", "<f8", 3), ("vel", "<f8", 3)])
    rec["type"] = system.type
    rec["mol"] = -1 if system.mol is None else system.mol
    rec["pos"] = system.pos
    rec["vel"] = system.vel
    with open(path, "wb") as f:
        f.write(np.int64(n).tobytes())
        f.write(rec.tobytes())


def read_blocks(path: str) -> Dict[str, np.ndarray]:
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        name = data[off:off + 16].split(b"\0", 1)[0].decode()
        count = int(np.frombuffer(data, np.int64, 1, off + 16)[0])
        elem = int(np.frombuffer(data, np.int32, 1, off + 24)[0])
        off += 32
        nbytes = count * elem
        dt = np.float64 if elem == 8 else np.int32
        arr = np.frombuffer(data, dt, count, off).copy()
        off += nbytes
        out[name] = arr[0] if count == 1 and name not in ("pairs", "sk") else arr
    if "pairs" in out:
        out["pairs"] = out["pairs"].reshape(-1, 5)
    for k in ("pos", "vel", "acc"):
        if k in out:
            out[k] = out[k].reshape(-1, 3)
    return out


def harness_available() -> bool:
    return os.path.exists(HARNESS_PATH)


def run_reference(system, mode: str = "forces", nsteps: int = 0, rebuild_test: bool = False,
                  timeout: Optional[float] = None, budget_s: float = 0.0, extra: str = "",
                  collect=(), mode_args=(), simulator: str = "basic",
                  harness: str = HARNESS_PATH) -> Dict[str, np.ndarray]:
    """Run the unmodified reference on `system` ("forces" or "run") and return
    its FP64 output blocks plus the harness's own wall time.  budget_s > 0
    stops a run after the step that crosses the budget (at least 2 steps).
    `extra` is appended to the script (e.g. writer objects); the text of the
    files named in `collect` (written by the reference in its working
    directory) comes back under "files".  Mode "runcall" calls the script's
    simulator's own run(); `simulator` names its class (e.g. "b200" with
    harness=HARNESS_B200_PATH, the reference built with the B200 integration
    layer)."""
    if not os.path.exists(harness):
        raise FileNotFoundError(f"reference harness not built: {harness}")
    with tempfile.TemporaryDirectory() as d:
        script = os.path.join(d, "sys.casl")
        state = os.path.join(d, "state.bin")
        out = os.path.join(d, "out.bin")
        with open(script, "w") as f:
            f.write(casl_script(system, nsteps, rebuild_test, extra, simulator))
        write_state(state, system)
        args = [harness, script, state, mode, out] + ([str(nsteps), repr(float(budget_s))] if mode == "run" else [])
        args += [str(x) for x in mode_args]  # e.g. randvel: seed, amplitude
        t0 = time.perf_counter()
        p = subprocess.run(args, cwd=d, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if p.returncode != 0 or not os.path.exists(out):
            raise RuntimeError(f"reference harness failed ({p.returncode}): {p.stdout[-2000:]}\n{p.stderr[-2000:]}")
        res = read_blocks(out)
        res["process_wall"] = wall
        files = {}
        for name in collect:
            fp = os.path.join(d, name)
            if os.path.exists(fp):
                with open(fp) as fh:
                    files[name] = fh.read()
        res["files"] = files
        return res
