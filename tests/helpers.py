"""Shared helpers for the parity tests: fixtures -> MDSystem, error metrics."""
import json
import os

import numpy as np

from caviar_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_path(name):
    return os.path.join(GOLDEN, name)


def load_ref_fixture(name):
    d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    T = len(d["mass"])
    lj = None
    if float(d["lj_cutoff"]) >= 0:
        cl = d["lj_cutoff_list"]
        lj = W.LJParams(cutoff=float(d["lj_cutoff"]), epsilon=d["lj_eps"], sigma=d["lj_sigma"],
                        cutoff_list=cl if cl.size else None)
    er = W.EwaldRParams(alpha=float(d["ewr_alpha"])) if float(d["ewr_alpha"]) >= 0 else None
    ek = W.EwaldKParams(alpha=float(d["ewk_alpha"]), kmax=tuple(int(x) for x in d["ewk_kmax"])) \
        if float(d["ewk_alpha"]) >= 0 else None
    s = W.MDSystem(lo=d["lo"], hi=d["hi"], mass=d["mass"], charge=d["charge"], pos=d["pos"], vel=d["vel"],
                   type=d["type"].astype(np.int32), cutoff=float(d["cutoff"]), coef=float(d["coef"]),
                   ghost_cutoff=float(d["ghost_cutoff"]), dt=float(d["dt"]), lj=lj, ewald_r=er, ewald_k=ek,
                   name=name)
    assert s.n_types == T
    return s, d


def ewald_golden():
    with open(os.path.join(GOLDEN, "ewald_n100.json")) as f:
        g = json.load(f)
    pos = np.array(g["pos"])
    n = len(pos)
    lo, hi = g["box"]
    kmax = int(g["kmax"])
    s = W.MDSystem(lo=np.full(3, lo), hi=np.full(3, hi), mass=np.array(g["mass_by_type"]),
                   charge=np.array(g["charge_by_type"]), pos=pos, vel=np.zeros((n, 3)),
                   type=np.array(g["type"], np.int32), cutoff=g["rcut"], coef=1.0, ghost_cutoff=g["rcut"], dt=0.001,
                   ewald_r=W.EwaldRParams(alpha=g["alpha"]),
                   ewald_k=W.EwaldKParams(alpha=g["alpha"], kmax=(kmax, kmax, kmax)), name="ewald_n100")
    return s, np.array(g["force"]), float(g["total_energy"])


def force_errors(f, ref):
    """(global ||dF|| / ||F||, max_i |dF_i| / rms|F|, median_i |dF_i| / |F_i|)."""
    d = np.linalg.norm(f - ref, axis=1)
    nref = np.linalg.norm(ref, axis=1)
    rms = np.sqrt(np.mean(nref ** 2))
    return (float(np.linalg.norm(d) / np.linalg.norm(nref)), float(d.max() / rms),
            float(np.median(d / np.maximum(nref, 1e-300))))
