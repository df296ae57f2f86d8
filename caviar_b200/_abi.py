"""ctypes binding of libcaviar_b200.so (the C ABI in include/caviar_b200.h).

`Simulation` wraps one context.  There is no fallback: if the library or a
CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CAVIAR_B200_LIB", os.path.join(HERE, "libcaviar_b200.so"))

OK = 0
ERR = {1: "INVALID", 2: "CUDA", 3: "NAN", 4: "STATE", 5: "GEOMETRY", 6: "CAPACITY", 7: "NOMEM"}
PREC_MIXED, PREC_FP64 = 0, 1
RNG_REFERENCE, RNG_PHILOX = 0, 1
DIPOLE_OFF, DIPOLE_REFERENCE, DIPOLE_ONCE = 0, 1, 2
REBUILD_DISPLACEMENT, REBUILD_REFERENCE, REBUILD_EVERY_STEP = 0, 1, 2
TH_KEYS = ["step", "ke", "temperature", "e_lj", "e_ewald_r", "e_ewald_k", "e_self", "virial", "pressure", "builds"]
N_THERMO = len(TH_KEYS)
KT_PAIR, KT_KSPACE, KT_INTEGRATE, KT_BUILD = 0, 1, 2, 3
LIST_AUTO, LIST_THREAD, LIST_WARP = 0, 1, 2
KFORCE_AUTO, KFORCE_CUDA_CORES = 0, 1

# Every symbol declared in include/caviar_b200.h.
EXPORTED = ["cvr_create", "cvr_destroy", "cvr_set_neighborlist", "cvr_set_lj", "cvr_set_ewald_r", "cvr_set_ewald_k",
            "cvr_set_integrator", "cvr_set_langevin", "cvr_set_berendsen", "cvr_set_nose_hoover",
            "cvr_clear_thermostat", "cvr_set_ewald_k_geometry",
            "cvr_set_ewald_slab_correction", "cvr_set_precision", "cvr_set_list_kernel", "cvr_set_kspace_force_kernel", "cvr_set_state", "cvr_build_neighbors", "cvr_compute_forces",
            "cvr_run", "cvr_get_state", "cvr_get_pairs", "cvr_get_sk", "cvr_get_scalars", "cvr_last_error",
            "cvr_launch_count", "cvr_get_stream", "cvr_get_info", "cvr_set_kernel_timing", "cvr_kernel_time",
            "cvr_structure_factor_noalloc", "cvr_casl_run_file", "cvr_batch_create", "cvr_batch_destroy",
            "cvr_batch_set_forces", "cvr_batch_set_state", "cvr_batch_run", "cvr_batch_get_state", "cvr_batch_info",
            "cvr_batch_last_error", "cvr_batch_stream", "cvr_adj_create", "cvr_adj_destroy", "cvr_adj_set_params",
            "cvr_adj_set_state", "cvr_adj_forces", "cvr_adj_force_vjp", "cvr_adj_loss", "cvr_adj_loss_grad",
            "cvr_adj_last_error", "cvr_adj_stream", "cvr_measure_fma_peak", "cvr_set_lj_jump_tol",
            "cvr_set_all_atom_test"]

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lib = None


class CvrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"CVR_ERR_{ERR.get(code, code)}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the library (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built; run python -m caviar_b200.build")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.cvr_create.argtypes = [ctypes.POINTER(vp), _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, _dp, _dp,
                             ctypes.c_int]
    L.cvr_destroy.argtypes = [vp]
    L.cvr_destroy.restype = None
    L.cvr_set_neighborlist.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    L.cvr_set_lj.argtypes = [vp, ctypes.c_double, _dp, _dp, _dp, ctypes.c_int]
    L.cvr_set_ewald_r.argtypes = [vp, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_double]
    L.cvr_set_ewald_k.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    L.cvr_set_integrator.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.cvr_set_langevin.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_uint64]
    L.cvr_set_precision.argtypes = [vp, ctypes.c_int]
    L.cvr_set_list_kernel.argtypes = [vp, ctypes.c_int]
    L.cvr_set_kspace_force_kernel.argtypes = [vp, ctypes.c_int]
    L.cvr_set_berendsen.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double]
    L.cvr_set_nose_hoover.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double]
    L.cvr_clear_thermostat.argtypes = [vp]
    L.cvr_set_ewald_k_geometry.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double]
    L.cvr_set_ewald_slab_correction.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_double]
    L.cvr_set_state.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp]
    L.cvr_build_neighbors.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.cvr_compute_forces.argtypes = [vp, vp, _dp]
    L.cvr_run.argtypes = [vp, ctypes.c_int64, ctypes.c_int64, _dp]
    L.cvr_get_state.argtypes = [vp, vp, vp, vp]
    L.cvr_get_pairs.argtypes = [vp, _ip]
    L.cvr_get_pairs.restype = ctypes.c_int64
    L.cvr_get_sk.argtypes = [vp, _dp]
    L.cvr_get_sk.restype = ctypes.c_int64
    L.cvr_get_scalars.argtypes = [vp, _dp]
    L.cvr_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.cvr_launch_count.argtypes = [vp]
    L.cvr_launch_count.restype = ctypes.c_int64
    L.cvr_get_stream.argtypes = [vp]
    L.cvr_get_stream.restype = vp
    L.cvr_get_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
    L.cvr_set_kernel_timing.argtypes = [vp, ctypes.c_int]
    L.cvr_kernel_time.argtypes = [vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int64)]
    L.cvr_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
    L.cvr_set_lj_jump_tol.argtypes = [vp, ctypes.c_double]
    L.cvr_set_all_atom_test.argtypes = [vp, ctypes.c_int]
    _lib = L
    return L


def fma_peak(device: int = 0, fp64: bool = False, iters: int = 2000):
    """(TFLOP/s, ms) of the FMA-only peak kernel (cvr_measure_fma_peak)."""
    L = load()
    tf, ms = ctypes.c_double(0), ctypes.c_double(0)
    rc = L.cvr_measure_fma_peak(device, int(fp64), iters, ctypes.byref(tf), ctypes.byref(ms))
    if rc != OK:
        raise CvrError(rc, "cvr_measure_fma_peak failed")
    return tf.value, ms.value


def run_casl(path: str) -> None:
    """Run a CASL script on the GPU (cvr_casl_run_file); raises on error."""
    L = load()
    f = L.cvr_casl_run_file
    f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
    f.restype = ctypes.c_int
    buf = ctypes.create_string_buffer(1024)
    rc = f(path.encode(), buf, 1024)
    if rc != OK:
        raise CvrError(rc, buf.value.decode(errors="replace"))


def _d(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(_dp)


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Simulation:
    """One periodic system on one GPU, driven through the C ABI."""

    def __init__(self, system=None, *, precision: int = PREC_MIXED, policy: int = REBUILD_DISPLACEMENT,
                 device: int = 0, lo=None, hi=None, bc=(1, 1, 1), mass=None, charge=None,
                 list_kernel: int = LIST_AUTO):
        self.L = load()
        if system is not None:
            lo, hi, bc, mass, charge = system.lo, system.hi, system.bc, system.mass, system.charge
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        charge = np.ascontiguousarray(np.zeros_like(mass) if charge is None else charge, np.float64)
        self.n_types = len(mass)
        h = ctypes.c_void_p()
        bca = (ctypes.c_int * 3)(*[int(b) for b in bc])
        rc = self.L.cvr_create(ctypes.byref(h), _d(lo), _d(hi), bca, self.n_types, _d(mass), _d(charge), device)
        if rc != OK:
            raise CvrError(rc, "cvr_create failed")
        self.h = h
        self.n = 0
        self._check(self.L.cvr_set_precision(self.h, precision))
        self._check(self.L.cvr_set_list_kernel(self.h, list_kernel))
        if system is not None:
            self.configure(system, policy)
            self.set_state(system.pos, system.vel, system.type, system.mol)

    # -- plumbing
    def _check(self, rc):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            self.L.cvr_last_error(self.h, buf, 512)
            raise CvrError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.L.cvr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- settings
    def configure(self, s, policy: int = REBUILD_DISPLACEMENT):
        self._check(self.L.cvr_set_neighborlist(self.h, s.cutoff, s.coef, s.ghost_cutoff, policy))
        if s.lj is not None:
            cl = None if s.lj.cutoff_list is None else s.lj.cutoff_list
            self._check(self.L.cvr_set_lj(self.h, s.lj.cutoff, _d(s.lj.epsilon), _d(s.lj.sigma), _d(cl),
                                          int(s.lj.ignore_intra_molecule)))
        if s.lj is not None and getattr(s.lj, "jump_tol", 0.0) > 0:
            self._check(self.L.cvr_set_lj_jump_tol(self.h, s.lj.jump_tol))
        if s.ewald_r is not None:
            self._check(self.L.cvr_set_ewald_r(self.h, s.ewald_r.alpha, s.ewald_r.k_electrostatic,
                                               _d(s.ewald_r.lam), s.ewald_r.cutoff))
        if s.ewald_k is not None:
            kx, ky, kz = s.ewald_k.kmax
            self._check(self.L.cvr_set_ewald_k(self.h, s.ewald_k.alpha, kx, ky, kz, s.ewald_k.k_electrostatic))
        self._check(self.L.cvr_set_integrator(self.h, s.dt, s.k_b))

    def set_integrator(self, dt: float, k_b: float = 1.0):
        """md_simulator dt / atom_data k_b (md_simulator.cpp:58-233)."""
        self._check(self.L.cvr_set_integrator(self.h, dt, k_b))

    def set_all_atom_test(self, on: bool = True):
        """neighborlist all_atom_test (neighborlist.cpp:161-191): every owned pair and ghost image."""
        self._check(self.L.cvr_set_all_atom_test(self.h, int(on)))

    def set_langevin(self, temperature: float, friction: float, kb: float = -1.0, kbt: float = -1.0,
                     rng: int = RNG_REFERENCE, seed: int = 0):
        """integrator_type velocity_verlet_langevin (md_simulator.cpp:670-811)."""
        self._check(self.L.cvr_set_langevin(self.h, temperature, friction, kb, kbt, rng, seed))

    def set_ewald_k_geometry(self, slab_axis: int = -1, slab_lz: float = 1.0, dipole_mode: int = DIPOLE_OFF,
                             epsilon_dipole: float = 0.0):
        """Electrostatic_ewald_k slab_normal_axis / slab_lz / epsilon_dipole."""
        self._check(self.L.cvr_set_ewald_k_geometry(self.h, slab_axis, slab_lz, dipole_mode, epsilon_dipole))

    def set_ewald_slab_correction(self, slab_axis: int, lz: float, kx_max: int, ky_max: int, k_e: float = 1.0):
        """force_field electrostatic_ewald_slab_correction."""
        self._check(self.L.cvr_set_ewald_slab_correction(self.h, slab_axis, lz, kx_max, ky_max, k_e))

    def set_berendsen(self, temperature: float, coupling: float, dt: float, step: int = 1, lambda_min: float = 0.8,
                      lambda_max: float = 1.25):
        """constraint berendsen (constraint/berendsen.cpp:44-131), defaults from berendsen.h:50-60."""
        self._check(self.L.cvr_set_berendsen(self.h, temperature, coupling, dt, step, lambda_min, lambda_max))

    def set_nose_hoover(self, temperature: float, dt: float, type: int = 1, mass: float = -1.0, tau: float = -1.0,
                        kb: float = 1.0):
        """constraint nose_hoover (constraint/nose_hoover.cpp:36-180)."""
        self._check(self.L.cvr_set_nose_hoover(self.h, temperature, type, mass, tau, kb, dt))

    def set_state(self, pos, vel=None, typ=None, mol=None):
        pos = np.ascontiguousarray(pos, np.float64)
        n = pos.shape[0]
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64)
        typ = np.ascontiguousarray(np.zeros(n, np.int32) if typ is None else typ, np.int32)
        mol = None if mol is None else np.ascontiguousarray(mol, np.int32)
        self._check(self.L.cvr_set_state(self.h, n, _ptr(pos), _ptr(vel), _ptr(typ), _ptr(mol)))
        self.n = n

    def set_state_ptr(self, n, pos_ptr, vel_ptr, type_ptr, mol_ptr=None):
        """Host pointers (e.g. pinned torch tensors) without numpy copies."""
        self._check(self.L.cvr_set_state(self.h, n, ctypes.c_void_p(pos_ptr), ctypes.c_void_p(vel_ptr),
                                         ctypes.c_void_p(type_ptr), None if mol_ptr is None else ctypes.c_void_p(mol_ptr)))
        self.n = n

    # -- hot path
    def build_neighbors(self, force: bool = True) -> bool:
        r = ctypes.c_int(0)
        self._check(self.L.cvr_build_neighbors(self.h, int(force), ctypes.byref(r)))
        return bool(r.value)

    def compute_forces(self):
        acc = np.zeros((self.n, 3))
        th = np.zeros(N_THERMO)
        self._check(self.L.cvr_compute_forces(self.h, _ptr(acc), _d(th)))
        return acc, dict(zip(TH_KEYS, th.tolist()))

    def run(self, nsteps: int, thermo_every: int = 0):
        nrec = nsteps // thermo_every if thermo_every > 0 else 0
        th = np.zeros((max(nrec, 1), N_THERMO))
        self._check(self.L.cvr_run(self.h, nsteps, thermo_every, th.ctypes.data_as(_dp)))
        return th[:nrec]

    def run_ptr(self, nsteps: int, thermo_every: int, thermo_ptr: Optional[int]):
        self._check(self.L.cvr_run(self.h, nsteps, thermo_every,
                                   None if thermo_ptr is None else ctypes.cast(thermo_ptr, _dp)))

    # -- readback
    def state(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        acc = np.zeros((self.n, 3))
        self._check(self.L.cvr_get_state(self.h, _ptr(pos), _ptr(vel), _ptr(acc)))
        return pos, vel, acc

    def get_state_ptr(self, pos_ptr, vel_ptr, acc_ptr):
        self._check(self.L.cvr_get_state(self.h, ctypes.c_void_p(pos_ptr) if pos_ptr else None,
                                         ctypes.c_void_p(vel_ptr) if vel_ptr else None,
                                         ctypes.c_void_p(acc_ptr) if acc_ptr else None))

    def pairs(self) -> np.ndarray:
        m = self.L.cvr_get_pairs(self.h, None)
        if m < 0:
            self._check(int(-m))
        out = np.zeros((m, 5), np.int32)
        m2 = self.L.cvr_get_pairs(self.h, out.ctypes.data_as(_ip))
        if m2 < 0:
            self._check(int(-m2))
        return out

    def sk(self) -> np.ndarray:
        m = self.L.cvr_get_sk(self.h, None)
        out = np.zeros((max(m, 0), 2))
        if m > 0:
            self.L.cvr_get_sk(self.h, out.ctypes.data_as(_dp))
        return out[:, 0] + 1j * out[:, 1]

    def scalars(self) -> dict:
        th = np.zeros(N_THERMO)
        self._check(self.L.cvr_get_scalars(self.h, th.ctypes.data_as(_dp)))
        return dict(zip(TH_KEYS, th.tolist()))

    def info(self) -> dict:
        v = (ctypes.c_int64 * 15)()
        self._check(self.L.cvr_get_info(self.h, v, 15))
        keys = ["n", "ncx", "ncy", "ncz", "cap", "builds", "tpa", "nk", "R", "max_count", "err", "step",
                "list_entries", "fixed_point", "kspace_tensor_cores"]
        return dict(zip(keys, list(v)))

    @property
    def launches(self) -> int:
        return int(self.L.cvr_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(self.L.cvr_get_stream(self.h) or 0)

    def set_kspace_force_kernel(self, kind: int):
        """KFORCE_AUTO (tensor cores where they apply) or KFORCE_CUDA_CORES."""
        self._check(self.L.cvr_set_kspace_force_kernel(self.h, kind))

    def set_kernel_timing(self, on: bool):
        self._check(self.L.cvr_set_kernel_timing(self.h, int(on)))

    def kernel_time(self, kind: int):
        ms = ctypes.c_double(0)
        n = ctypes.c_int64(0)
        self._check(self.L.cvr_kernel_time(self.h, kind, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value


class Batch:
    """Many small periodic replicas on one GPU (cvr_batch_* of the C ABI)."""

    N_OUT = 8
    OUT_KEYS = ["ke", "e_lj", "e_ewald_r", "e_ewald_k", "e_self", "virial", "temperature", "steps"]

    def __init__(self, n_atoms, box, mass, charge, device: int = 0):
        L = load()
        vp = ctypes.c_void_p
        L.cvr_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int]
        L.cvr_batch_destroy.argtypes = [vp]
        L.cvr_batch_destroy.restype = None
        L.cvr_batch_set_forces.argtypes = [vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double]
        L.cvr_batch_set_state.argtypes = [vp, vp, vp, vp]
        L.cvr_batch_run.argtypes = [vp, ctypes.c_int64, vp]
        L.cvr_batch_get_state.argtypes = [vp, vp, vp, vp]
        L.cvr_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.cvr_batch_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.cvr_batch_stream.argtypes = [vp]
        L.cvr_batch_stream.restype = vp
        self.L = L
        self.n = np.ascontiguousarray(n_atoms, np.int64)
        self.box = np.ascontiguousarray(box, np.float64)
        self.n_rep = len(self.n)
        self.n_total = int(self.n.sum())
        m = np.ascontiguousarray(mass, np.float64)
        q = np.ascontiguousarray(charge, np.float64)
        h = vp()
        rc = L.cvr_batch_create(ctypes.byref(h), self.n_rep, _ptr(self.n), _ptr(self.box), len(m), _ptr(m), _ptr(q),
                                device)
        if rc != OK:
            raise CvrError(rc, "cvr_batch_create failed")
        self.h = h

    def _check(self, rc):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            self.L.cvr_batch_last_error(self.h, buf, 512)
            raise CvrError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.L.cvr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_forces(self, eps, sigma, rc_lj, rc_r, alpha, kmax, k_e=1.0, dt=0.005):
        self._keep = [np.ascontiguousarray(x, np.float64) for x in (eps, sigma, rc_lj, rc_r)]
        e, sg, rl, rr = self._keep
        self._check(self.L.cvr_batch_set_forces(self.h, _ptr(e), _ptr(sg), _ptr(rl), _ptr(rr), alpha, kmax, k_e, dt))

    def set_state(self, pos, vel, typ):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        typ = np.ascontiguousarray(typ, np.int32)
        self._check(self.L.cvr_batch_set_state(self.h, _ptr(pos), _ptr(vel), _ptr(typ)))

    def run(self, nsteps: int):
        out = np.zeros((self.n_rep, self.N_OUT))
        self._check(self.L.cvr_batch_run(self.h, nsteps, _ptr(out)))
        return out

    def state(self):
        pos = np.zeros((self.n_total, 3))
        vel = np.zeros((self.n_total, 3))
        acc = np.zeros((self.n_total, 3))
        self._check(self.L.cvr_batch_get_state(self.h, _ptr(pos), _ptr(vel), _ptr(acc)))
        return pos, vel, acc

    def info(self):
        v = (ctypes.c_int64 * 64)()
        self._check(self.L.cvr_batch_info(self.h, v, 64))
        n_cls = int(v[2])
        classes = [dict(replicas=int(v[3 + 4 * c]), nmax=int(v[4 + 4 * c]), threads=int(v[5 + 4 * c]),
                        sk_groups=int(v[6 + 4 * c])) for c in range(n_cls)]
        return {"n_rep": int(v[0]), "atoms": int(v[1]), "classes": classes}

    @property
    def stream(self) -> int:
        return int(self.L.cvr_batch_stream(self.h) or 0)


class Adjoint:
    """Trajectory-loss gradient on the GPU (cvr_adj_* of the C ABI).

    theta vectors are laid out eps[T*T], sigma[T*T], charge[T]."""

    def __init__(self, n: int, box: float, mass, precision: int = PREC_MIXED, device: int = 0):
        L = load()
        vp, dp = ctypes.c_void_p, ctypes.c_double
        L.cvr_adj_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int64, dp, ctypes.c_int, vp, ctypes.c_int,
                                     ctypes.c_int]
        L.cvr_adj_destroy.argtypes = [vp]
        L.cvr_adj_destroy.restype = None
        L.cvr_adj_set_params.argtypes = [vp, vp, vp, vp, dp, dp, dp, ctypes.c_int, dp, dp]
        L.cvr_adj_set_state.argtypes = [vp, vp, vp, vp]
        L.cvr_adj_forces.argtypes = [vp, vp, vp, vp]
        L.cvr_adj_force_vjp.argtypes = [vp, vp, vp, vp]
        L.cvr_adj_loss.argtypes = [vp, ctypes.c_int64, vp, vp, vp]
        L.cvr_adj_loss_grad.argtypes = [vp, ctypes.c_int64, ctypes.c_int64, vp, vp, vp, vp]
        L.cvr_adj_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.cvr_adj_stream.argtypes = [vp]
        L.cvr_adj_stream.restype = vp
        self.L = L
        self.n = int(n)
        m = np.ascontiguousarray(mass, np.float64)
        self.nt = len(m)
        h = vp()
        rc = L.cvr_adj_create(ctypes.byref(h), self.n, float(box), self.nt, _ptr(m), precision, device)
        if rc != OK:
            raise CvrError(rc, "cvr_adj_create failed")
        self.h = h

    @classmethod
    def from_system(cls, s, precision: int = PREC_MIXED, device: int = 0) -> "Adjoint":
        """From a workloads.AdjointSystem: parameters and initial state set."""
        a = cls(len(s.pos), s.box, s.mass, precision, device)
        a.set_params(s.charge, s.epsilon, s.sigma, s.rc_lj, s.alpha, s.rc_r, s.kmax, s.k_e, s.dt)
        a.set_state(s.pos, s.vel, s.type)
        return a

    def _check(self, rc):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            self.L.cvr_adj_last_error(self.h, buf, 512)
            raise CvrError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.L.cvr_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def split(self, g):
        t = self.nt
        return {"eps": g[:t * t].reshape(t, t), "sigma": g[t * t:2 * t * t].reshape(t, t), "charge": g[2 * t * t:]}

    def set_params(self, charge, eps, sigma, rc_lj, alpha, rc_r, kmax, k_e=1.0, dt=0.002):
        q, e, sg = (np.ascontiguousarray(x, np.float64) for x in (charge, eps, sigma))
        self._check(self.L.cvr_adj_set_params(self.h, _ptr(q), _ptr(e), _ptr(sg), rc_lj, alpha, rc_r, kmax, k_e, dt))

    def set_state(self, pos, vel, typ):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        typ = np.ascontiguousarray(typ, np.int32)
        self._check(self.L.cvr_adj_set_state(self.h, _ptr(pos), _ptr(vel), _ptr(typ)))

    def forces(self):
        f, e, g = np.zeros((self.n, 3)), np.zeros(4), np.zeros(2 * self.nt * self.nt + self.nt)
        self._check(self.L.cvr_adj_forces(self.h, _ptr(f), _ptr(e), _ptr(g)))
        return f, e, self.split(g)

    def force_vjp(self, u):
        u = np.ascontiguousarray(u, np.float64)
        w, g = np.zeros((self.n, 3)), np.zeros(2 * self.nt * self.nt + self.nt)
        self._check(self.L.cvr_adj_force_vjp(self.h, _ptr(u), _ptr(w), _ptr(g)))
        return w, self.split(g)

    def loss(self, nsteps: int):
        J = np.zeros(1)
        self._check(self.L.cvr_adj_loss(self.h, nsteps, _ptr(J), None, None))
        return float(J[0])

    def loss_grad(self, nsteps: int, checkpoint_every: int = 50):
        J = np.zeros(1)
        gp, gv = np.zeros((self.n, 3)), np.zeros((self.n, 3))
        g = np.zeros(2 * self.nt * self.nt + self.nt)
        self._check(self.L.cvr_adj_loss_grad(self.h, nsteps, checkpoint_every, _ptr(J), _ptr(gp), _ptr(gv), _ptr(g)))
        out = {"pos": gp, "vel": gv}
        out.update(self.split(g))
        return float(J[0]), out
