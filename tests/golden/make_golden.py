"""Generates the golden fixtures in this folder from the reference itself.

The reference's CPU code (GreedyIteratorCPU, LDMMIteratorCPU,
HField3DUtils, Array3DUtils, DiffOperT, GaussianFilter3D, ...) is compiled
from its own sources by oracle/ref/Makefile into oracle/_ref/libawref.so;
this script feeds it small seeded inputs and stores inputs and outputs as
compressed .npz files, so the parity tests can check both the oracle and
the CUDA path against reference outputs on machines without the reference
tree. Run from the repository root:

    python tests/golden/make_golden.py            (every fixture)
    python tests/golden/make_golden.py adshoot    (the adjoint-shooting ones)

Every case is deterministic (seeded numpy generators); re-running rewrites
identical files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from atlaswerks_b200.synth import atlas_subjects, bullseye, greedy_pair  # noqa: E402
from oracle import REF_SO, Reference, build_reference, identity, reference_root  # noqa: E402
from atlaswerks_b200.metaimage import read_mha, read_nhdr, rescale_intensities  # noqa: E402

BG = ["partial_id", "id", "partial_zero", "zero", "clamp", "wrap"]


def small_pair(shape, seed, n_blobs=6, umax=1.5):
    """A pair whose blobs are sized for a 16-voxel grid (no saturation)."""
    return greedy_pair(shape, seed, n_blobs, umax, sigma_range=(1.5, 3.0), smooth_sigma=3.0)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def main():
    if not os.path.exists(REF_SO) and not build_reference():
        raise SystemExit("the reference CPU build is needed (oracle/ref/Makefile)")
    ref = Reference()
    rng = np.random.default_rng(2024)

    # interpolation family on a ragged grid, spacing != 1
    shape = (9, 13, 11)
    sp = (1.5, 0.75, 1.25)
    img = rng.random(shape, dtype=np.float32)
    h = identity(shape) + rng.normal(0, 2.5, (3,) + shape).astype(np.float32)
    v = rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    out = dict(img=img, h=h, v=v, sp=np.array(sp), apply=ref.apply(img, h),
               gradient=ref.gradient(img, sp, False), gradient_wrap=ref.gradient(img, sp, True),
               splat=ref.splat(img, h))
    for b, name in enumerate(BG):
        out["compose_hv_" + name] = ref.compose_hv(h, v, sp, 1, b)
        out["compose_hvinv_" + name] = ref.compose_hv(h, v, sp, -1, b)
        out["compose_vhinv_" + name] = ref.compose_vh(v, h, sp, -1, b)
    save("interp_9x13x11", **out)

    # fluid operator (FP32 reference path through the FFTW-API shim), 16x12x20
    shape = (20, 12, 16)
    sp = (1.0, 1.25, 0.8)
    f = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    save("fluid_16x12x20", f=f, sp=np.array(sp), alpha=0.01, beta=0.01, gamma=0.001,
         inverse=ref.fluid(f, sp, 0.01, 0.01, 0.001, True),
         forward=ref.fluid(f, sp, 0.01, 0.01, 0.001, False),
         inverse_f64=ref.fluid_f64(f, sp, 0.01, 0.01, 0.001, True))

    # greedy: single scale 16^3 x 12 iterations, and two scales 32^3 (2, 1)
    I0, I1 = small_pair((16, 16, 16), 7)
    hh, hi, en, st = ref.greedy_run(I0, I1, [1], [12], [0.5], inverse=True)
    save("greedy_16", I0=I0, I1=I1, h=hh, hinv=hi, energies=en, steps=st)
    I0, I1 = greedy_pair((24, 24, 24), 8, 8, 2.0, sigma_range=(2.0, 4.0), smooth_sigma=4.0)
    hh, _, en, st = ref.greedy_run(I0, I1, [2, 1], [10, 6], [0.5, 0.5])
    save("greedy_24_two_scales", I0=I0, I1=I1, h=hh, energies=en, steps=st)

    # multiscale pieces
    img = bullseye((24, 20, 16), (7.0, 5.0, 3.0))
    save("downsample_16x20x24", img=img, half=ref.downsample(img, (12, 10, 8)))
    hf = identity((8, 10, 12)) + rng.normal(0, 0.7, (3, 8, 10, 12)).astype(np.float32)
    save("upsample_12x10x8", h=hf, up=ref.upsample_hfield(hf, (16, 20, 24), True),
         up_norescale=ref.upsample_hfield(hf, (16, 20, 24), False))

    # LDMM relaxation, IterateNew, 16^3, T = 4, fixed and adaptive steps
    I0, I1 = small_pair((16, 16, 16), 9)
    vv, en, stp = ref.ldmm_run(I0, I1, 4, 8, sigma=1.0, step=0.01)
    va, ea, sa = ref.ldmm_run(I0, I1, 4, 6, sigma=1.0, step=0.01, adaptive=True, max_pert=0.2)
    save("ldmm_16_T4", I0=I0, I1=I1, v=vv, energies=en, step=np.float32(stp), v_adaptive=va,
         energies_adaptive=ea, step_adaptive=np.float32(sa))

    # LDMM IterateOrig (Jacobian transport, the reference's default), 16x14x12,
    # T = 4, anisotropic spacing; fixed and adaptive steps
    I0, I1 = small_pair((12, 14, 16), 10)
    sp = (1.5, 0.75, 1.25)
    vo, eo, so = ref.ldmm_run(I0, I1, 4, 6, sp=sp, sigma=1.0, step=0.01, use_new=False)
    voa, eoa, soa = ref.ldmm_run(I0, I1, 4, 4, sp=sp, sigma=1.0, step=0.01, adaptive=True,
                                 max_pert=0.2, use_new=False)
    save("ldmm_orig_16x14x12_T4", I0=I0, I1=I1, sp=np.array(sp), v=vo, energies=eo,
         step=np.float32(so), v_adaptive=voa, energies_adaptive=eoa, step_adaptive=np.float32(soa))

    # greedy atlas, equal grids 16^3, 3 subjects, mean every iteration and every 2nd
    imgs = atlas_subjects(3, 13, sizes=(16,), n_blobs=6, umax=2.0)
    w = np.array([0.25, 0.35, 0.4], np.float32)
    m1, h1, e1 = ref.atlas_run(imgs, list(w), 6, 1)
    m2, h2, e2 = ref.atlas_run(imgs, list(w), 6, 2)
    save("atlas_16x3", imgs=np.stack(imgs), w=w, mean_p1=m1, h_p1=np.stack(h1), energies_p1=e1,
         mean_p2=m2, h_p2=np.stack(h2), energies_p2=e2)

    adshoot_cases(ref)
    greedy_bullseye_case(ref)


def adshoot_cases(ref):
    """LDMM adjoint shooting: a small single-scale run, and the reference's
    own regression (Testing/Applications/LDMM/LDMMAdShootingWarp: the
    bullseye pair rescaled to [0, 1], scale factors 2 then 1 with 100
    iterations each at steps 0.0005 / 0.0002, T = 5, sigma 1, alpha = beta =
    0.01, gamma = 0.001) with its Baseline deformed image."""
    I0, I1 = small_pair((12, 14, 16), 11)
    sp = (1.5, 0.75, 1.25)
    a0, p0, p1, ei, ev = ref.adshoot_run(I0, I1, 4, [(1, 5, 0.0002)], sp, sigma=1.0)
    save("adshoot_16x14x12_T4", I0=I0, I1=I1, sp=np.array(sp), alpha0=a0, phi0T=p0, phiT0=p1,
         img_energy=ei, vec_energy=ev)
    root = os.path.join(reference_root(), "Testing")
    B0, bsp = read_nhdr(f"{root}/Data/Input/Bullseyes/BullseyeTestBlur00.nhdr")
    B1, _ = read_nhdr(f"{root}/Data/Input/Bullseyes/BullseyeTestBlur01.nhdr")
    base, _ = read_mha(f"{root}/Applications/LDMM/LDMMAdShootingWarp/Baseline/"
                       "LDMMAdShootingWarpBullseyeTestBlur00_to_BullseyeTestBlur01DefImage.mha")
    B0, B1 = rescale_intensities(B0), rescale_intensities(B1)
    levels = [(1, 100, 0.0002), (2, 100, 0.0005)]
    a0, _, p1, ei, ev = ref.adshoot_run(B0, B1, 5, levels, bsp, sigma=1.0)
    save("adshoot_bullseye", I0=B0, I1=B1, sp=np.array(bsp), baseline_def_image=base,
         alpha0=a0, phiT0=p1, img_energy=ei, vec_energy=ev)


def greedy_bullseye_case(ref):
    """The reference's greedy regression (Testing/Applications/Greedy/
    GreedyWarp: GreedyWarpParams.xml — the bullseye pair rescaled to [0, 1],
    scale factors 2 then 1 with 50 iterations each, MaxPert 0.3, alpha =
    beta = 0.01, gamma = 0.001, the inverse field computed) with its
    Baseline deformed image, and the reference build's own run on it."""
    root = os.path.join(reference_root(), "Testing")
    B0, bsp = read_nhdr(f"{root}/Data/Input/Bullseyes/BullseyeTestBlur00.nhdr")
    B1, _ = read_nhdr(f"{root}/Data/Input/Bullseyes/BullseyeTestBlur01.nhdr")
    base, _ = read_mha(f"{root}/Applications/Greedy/GreedyWarp/Baseline/"
                       "GreedyBullseyeTestBlur00_to_BullseyeTestBlur01DefImage.mha")
    B0, B1 = rescale_intensities(B0), rescale_intensities(B1)
    h, hinv, en, steps = ref.greedy_run(B0, B1, [2, 1], [50, 50], [0.3, 0.3], bsp, inverse=True)
    save("greedy_bullseye", I0=B0, I1=B1, sp=np.array(bsp), baseline_def_image=base, h=h,
         hinv=hinv, energies=en)


if __name__ == "__main__":
    if sys.argv[1:] == ["adshoot"]:
        adshoot_cases(Reference())
    elif sys.argv[1:] == ["greedy_bullseye"]:
        greedy_bullseye_case(Reference())
    else:
        main()
