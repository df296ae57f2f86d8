"""The reference built with the B200 integration layer (caviar_b200/integration):
`md_simulator b200` / `b200_fp64` registered in the reference's own object
factory, its run() done through the C ABI inside the reference binary
(oracle/_ref/ref_harness_b200, made by oracle/Makefile's ref_b200 target from
the unmodified reference sources plus the adapter).

CPU: the factory knows the new class names and the adapter's run() is the
one the script reaches (without a GPU it stops in cvr_create with the
adapter's own message through the reference's error path); `md_simulator
basic` in the same binary is the reference's own run.
GPU: a script run with `md_simulator b200_fp64` (and `b200`) ends in the
state `md_simulator basic` reaches in the same binary: positions within
1e-9 (FP64) / 1e-5 (mixed) after 20 velocity-Verlet steps.
"""
import os

import numpy as np
import pytest

from helpers import load_ref_fixture


def harness(oracle_lib):
    if not os.path.exists(oracle_lib.HARNESS_B200_PATH):
        pytest.fail("oracle/_ref/ref_harness_b200 not built (oracle/Makefile ref_b200)")
    return oracle_lib.HARNESS_B200_PATH


def run(oracle_lib, s, simulator, nsteps=20):
    r = oracle_lib.run_reference(s, "runcall", nsteps=nsteps, simulator=simulator, harness=harness(oracle_lib),
                                 timeout=600)
    order = np.argsort(r["id"].astype(np.int64))
    return r["pos"].reshape(-1, 3)[order], r["vel"].reshape(-1, 3)[order], r["acc"].reshape(-1, 3)[order]


def test_factory_dispatches_to_the_adapter(oracle_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU failure path")
    s, _ = load_ref_fixture("lj500")
    with pytest.raises(RuntimeError) as e:
        run(oracle_lib, s, "b200", 2)
    assert "md_simulator b200" in str(e.value)
    pos, vel, acc = run(oracle_lib, s, "basic", 2)  # the reference's own run() in the same binary
    assert np.isfinite(pos).all() and pos.shape == (s.n, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lj500", "ions500"])
@pytest.mark.parametrize("simulator,tol", [("b200_fp64", 1e-9), ("b200", 1e-5)])
def test_b200_simulator_matches_basic(oracle_lib, name, simulator, tol):
    s, _ = load_ref_fixture(name)
    p0, v0, a0 = run(oracle_lib, s, "basic")
    p1, v1, a1 = run(oracle_lib, s, simulator)
    d = p1 - p0
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < tol, np.abs(d).max()
    assert np.abs(v1 - v0).max() < 100 * tol
    assert np.linalg.norm(a1 - a0) <= 100 * tol * np.linalg.norm(a0)
