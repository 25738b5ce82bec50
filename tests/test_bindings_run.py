"""The reference-side bindings (include/aw_b200_greedy_iterator.hpp,
aw_b200_ldmm_iterator.hpp, aw_b200_diffoper.hpp) compiled over stand-ins of
the few AtlasWerks headers they include (tests/binding/), linked against
libaw_b200.so and run the way GreedyWarp / LDMMWarp drive an iterator
(tests/binding/binding_driver.cpp).

* CPU: the driver compiles and links (every aw_* symbol the bindings call
  resolves in libaw_b200.so).
* GPU: the bindings' results equal the host mirror's over the same library
  bit for bit (fields, velocities, alphas, energies as float); the Jacobian
  equals the oracle's (bit-exact); DiffOperB200 is within 1e-5 of max |fp64|.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "atlaswerks_b200")


def build_driver(out_dir):
    exe = os.path.join(str(out_dir), "binding_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "tests", "binding"),
           "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "binding", "binding_driver.cpp"), "-L", LIB_DIR,
           "-law_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{LIB_DIR}",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_bindings_compile_and_link(tmp_path):
    if not os.path.exists(os.path.join(LIB_DIR, "libaw_b200.so")):
        pytest.skip("libaw_b200.so not built")
    assert os.path.exists(build_driver(tmp_path))


def _run(exe, *args):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


def _raw(path, shape):
    return np.fromfile(path, dtype=np.float32).reshape(shape)


@pytest.mark.gpu
@pytest.mark.parametrize("inverse", [False, True])
def test_greedy_binding_equals_host_mirror(tmp_path, inverse):
    import torch

    from atlaswerks_b200.greedy import (DiffOperParam, GreedyDeformationDataB200,
                                        GreedyIteratorB200, GreedyIteratorParam)
    from atlaswerks_b200.synth import greedy_pair
    shape, iters = (32, 32, 32), 6
    I0, I1 = greedy_pair(shape, seed=61, n_blobs=6, umax=2.0)
    I0.tofile(tmp_path / "I0.raw")
    I1.tofile(tmp_path / "I1.raw")
    _run(build_driver(tmp_path), "greedy", tmp_path, 32, 32, 32, iters, int(inverse))
    it = GreedyIteratorB200((32, 32, 32))
    it.SetScaleLevel((32, 32, 32), (1.0, 1.0, 1.0), GreedyIteratorParam(DiffOperParam(), 0.5))
    d = GreedyDeformationDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda(),
                                  compute_inverse=inverse)
    it.UpdateStepSizeNextIteration()
    for _ in range(iters):
        it.Iterate(d)
    torch.cuda.synchronize()
    assert np.array_equal(_raw(tmp_path / "h.raw", (3,) + shape), d.Def1To0().cpu().numpy())
    if inverse:
        assert np.array_equal(_raw(tmp_path / "hinv.raw", (3,) + shape),
                              d.Def0To1().cpu().numpy())
    e = np.fromfile(tmp_path / "energies.raw", dtype=np.float32)
    assert np.array_equal(e, it.Energies().astype(np.float32))
    assert np.fromfile(tmp_path / "step.raw", dtype=np.float32)[0] == np.float32(it.StepSize())


@pytest.mark.gpu
def test_ldmm_binding_equals_host_mirror(tmp_path, oracle):
    import torch

    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.ldmm import (LDMMDeformationDataB200, LDMMIteratorB200,
                                      LDMMIteratorParam, ldmm_total_energy)
    from atlaswerks_b200.synth import greedy_pair
    shape, T, iters = (16, 16, 16), 3, 4
    n = 16 ** 3
    I0, I1 = greedy_pair(shape, seed=62, n_blobs=4, umax=2.0)
    I0.tofile(tmp_path / "I0.raw")
    I1.tofile(tmp_path / "I1.raw")
    _run(build_driver(tmp_path), "ldmm", tmp_path, 16, 16, 16, T, iters)
    it = LDMMIteratorB200((16, 16, 16), n_time_steps=T)
    it.SetVectorEnergy(True)  # the binding's debug mode records them
    it.SetScaleLevel((16, 16, 16), (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, False, 0.1))
    d = LDMMDeformationDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda(), T)
    totals = []
    for _ in range(iters):
        it.Iterate(d)
        totals.append(it.TotalEnergy())
    torch.cuda.synchronize()
    v = d.V.cpu().numpy()
    assert np.array_equal(_raw(tmp_path / "v.raw", (T, 3) + shape), v)
    it.Iterate(d, computeAlphasOnly=True)
    al = np.stack([it.GetAlpha(t).cpu().numpy() for t in range(T)])
    assert np.array_equal(_raw(tmp_path / "alphas.raw", (T,) + shape), al)
    _, jd = oracle.ldmm_i1_at_0(I1, v)
    assert np.array_equal(_raw(tmp_path / "jacdet.raw", shape), jd)
    e = np.fromfile(tmp_path / "energies.raw", dtype=np.float32)
    # LDMMEnergy::GetEnergy: image / sigma^2 + the step energies' mean (the
    # alphas-only pass records the image term only)
    totals.append(ldmm_total_energy(it.Energies()[-1], np.zeros(T), 1.0, T))
    assert len(e) == iters + 1 and np.array_equal(e, np.array(totals, np.float32))
    assert all(t > it.Energies()[k] for k, t in enumerate(totals[:iters]))
    assert n == v[0, 0].size


@pytest.mark.gpu
@pytest.mark.parametrize("inverse", [True, False])
def test_diffoper_binding_vs_fp64(tmp_path, oracle, inverse):
    shape = (20, 24, 32)  # (nz, ny, nx)
    rng = np.random.default_rng(63)
    f = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    f.tofile(tmp_path / "f.raw")
    _run(build_driver(tmp_path), "diffoper", tmp_path, 32, 24, 20, int(inverse))
    got = _raw(tmp_path / "out.raw", (3,) + shape).astype(np.float64)
    want = oracle.fluid_f64(f, (1.0, 1.3, 0.8), inverse=inverse)
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-5
