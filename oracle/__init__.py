"""Test oracle for the greedy-fluid / LDMM inner loop.

TEST INFRASTRUCTURE. Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this package; the product package
``atlaswerks_b200`` never does.

Two libraries are wrapped, both taking planar float32 numpy arrays:

* ``Oracle`` — ``oracle/liboracle.so``, the C restatement of the reference
  CPU routines (``oracle/aw_oracle.c``), with the fluid operator in FP64.
* ``Reference`` — ``oracle/_ref/libawref.so``, the reference's own CPU code
  (``GreedyIteratorCPU``, ``HField3DUtils``, ``DiffOperT``) compiled from its
  sources by ``oracle/ref/Makefile``. It pins the oracle; it exists where the
  reference tree was present at build time (its ``.so`` travels with the
  repository snapshot).
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import subprocess
import sys
import threading
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libawref.so")

# HField3DUtils::VectorBackgroundStrategy (UtilitiesDataTypes/HField3DUtils.h:44-49)
BG_PARTIAL_ID, BG_ID, BG_PARTIAL_ZERO, BG_ZERO, BG_CLAMP, BG_WRAP = range(6)

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.c_int
_dbl = ctypes.c_double


def _fp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_f)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_d)


def build_oracle() -> None:
    """Compile liboracle.so (gcc only; no reference tree needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def reference_root() -> str:
    """Root of the reference source tree: $AW_REFERENCE_ROOT when set, else
    the read-only checkout this build was developed against."""
    return os.environ.get("AW_REFERENCE_ROOT", "/root/reference")


def build_reference(ref_root: Optional[str] = None) -> bool:
    """Compile the reference CPU path into _ref/libawref.so when the
    reference tree is present. Returns True when the library exists."""
    ref_root = ref_root or reference_root()
    if os.path.isdir(ref_root):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), f"REF={ref_root}"],
                       check=True)
    return os.path.exists(REF_SO)


def _shape(a: np.ndarray):
    nz, ny, nx = a.shape[-3:]
    return nx, ny, nz


def identity(shape) -> np.ndarray:
    """Identity h-field, planar [3, nz, ny, nx] (x, y, z components)."""
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([x, y, z]).astype(np.float32)


class Oracle:
    """ctypes wrapper of liboracle.so (arrays are [nz, ny, nx], fields [3, nz, ny, nx])."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.aw_oracle_greedy_iterate.restype = ctypes.c_double
        L.aw_oracle_max_norm.restype = ctypes.c_float
        L.aw_oracle_ldmm_iterate.restype = ctypes.c_double
        L.aw_oracle_atlas_iterate.restype = ctypes.c_double
        L.aw_oracle_ldmm_iterate_orig.restype = ctypes.c_double
        L.aw_oracle_ldmm_velshoot_iterate.restype = ctypes.c_double
        L.aw_oracle_ldmm_shoot_iterate.restype = ctypes.c_double
        L.aw_oracle_ldmm_adshoot_iterate.restype = ctypes.c_double

    # --- interpolation family -------------------------------------------------
    def apply(self, img, h, bg=0.0):
        out = np.empty_like(img)
        self.lib.aw_oracle_apply(_fp(img), _fp(h[0]), _fp(h[1]), _fp(h[2]), _fp(out),
                                 *_shape(img), ctypes.c_float(bg))
        return out

    def apply_u(self, img, v, sp=(1.0, 1.0, 1.0), bg=0.0):
        out = np.empty_like(img)
        self.lib.aw_oracle_apply_u(_fp(img), _fp(v[0]), _fp(v[1]), _fp(v[2]), _fp(out),
                                   *_shape(img), *map(_dbl, sp), ctypes.c_float(bg))
        return out

    def gradient(self, img, sp=(1.0, 1.0, 1.0), wrap=False):
        g = np.zeros((3,) + img.shape, np.float32)
        self.lib.aw_oracle_gradient(_fp(img), _fp(g[0]), _fp(g[1]), _fp(g[2]), *_shape(img),
                                    *map(_dbl, sp), _i(int(wrap)))
        return g

    def compose_hv(self, g, v, sp=(1.0, 1.0, 1.0), direction=1, bg=BG_PARTIAL_ID):
        o = np.empty_like(g)
        self.lib.aw_oracle_compose_hv(_fp(g[0]), _fp(g[1]), _fp(g[2]), _fp(v[0]), _fp(v[1]),
                                      _fp(v[2]), _fp(o[0]), _fp(o[1]), _fp(o[2]), *_shape(g),
                                      *map(_dbl, sp), _i(direction), _i(bg))
        return o

    def compose_vh(self, v, g, sp=(1.0, 1.0, 1.0), direction=-1, bg=BG_PARTIAL_ZERO):
        o = np.empty_like(g)
        self.lib.aw_oracle_compose_vh(_fp(v[0]), _fp(v[1]), _fp(v[2]), _fp(g[0]), _fp(g[1]),
                                      _fp(g[2]), _fp(o[0]), _fp(o[1]), _fp(o[2]), *_shape(g),
                                      *map(_dbl, sp), _i(direction), _i(bg))
        return o

    def splat(self, img, h, bg=0.0):
        out = np.empty_like(img)
        self.lib.aw_oracle_splat(_fp(img), _fp(h[0]), _fp(h[1]), _fp(h[2]), _fp(out),
                                 *_shape(img), ctypes.c_float(bg))
        return out

    # --- fluid operator ---------------------------------------------------------
    def fluid(self, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001, inverse=True):
        """L^-1 v (inverse) or L v in FP64; float32 in -> float32 out."""
        o = np.ascontiguousarray(v, dtype=np.float32).copy()
        self.lib.aw_oracle_fluid_apply(_fp(o[0]), _fp(o[1]), _fp(o[2]), *_shape(o),
                                       *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
                                       _i(int(inverse)))
        return o

    def fluid_f64(self, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001, inverse=True):
        o = np.ascontiguousarray(v, dtype=np.float64).copy()
        self.lib.aw_oracle_fluid_apply_f64(_dp(o[0]), _dp(o[1]), _dp(o[2]), *_shape(o),
                                           *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
                                           _i(int(inverse)))
        return o

    def downsample(self, img, new_shape, sp=(1.0, 1.0, 1.0)):
        """ImageUtils::gaussianDownsample to new_shape = (nz, ny, nx)."""
        out = np.empty(new_shape, np.float32)
        mz, my, mx = new_shape
        self.lib.aw_oracle_downsample(_fp(img), *_shape(img), *map(_dbl, sp), _fp(out),
                                      _i(mx), _i(my), _i(mz))
        return out

    def upsample_hfield(self, h, new_shape, rescale=True):
        out = np.empty((3,) + tuple(new_shape), np.float32)
        mz, my, mx = new_shape
        self.lib.aw_oracle_upsample_hfield(_fp(np.ascontiguousarray(h)), *_shape(h), _fp(out),
                                           _i(mx), _i(my), _i(mz), _i(int(rescale)))
        return out

    def greedy_warp(self, I0, I1, levels, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                    gamma=0.001, inverse=False):
        """Multiscale greedy (GreedyWarp::RunWarp); levels = [(factor, iters,
        max_pert)], any order. Returns (h, hinv, energies per level)."""
        levels = sorted(levels, key=lambda l: -l[0])
        shape = I0.shape
        h = hinv = None
        energies = []
        for li, (f, iters, mp) in enumerate(levels):
            size = tuple(n // f for n in shape)
            lsp = tuple(float(np.float32(s) * np.float32(f)) for s in sp)
            if size == tuple(shape):
                a, b = I0, I1
            else:
                a, b = self.downsample(I0, size, sp), self.downsample(I1, size, sp)
            if li == 0:
                h = identity(size)
                hinv = identity(size) if inverse else None
            else:
                h = self.upsample_hfield(h, size, True)
                hinv = self.upsample_hfield(hinv, size, True) if inverse else None
            step, es = 0.0, []
            for it in range(iters):
                e, step = self.greedy_iterate(a, b, h, hinv, lsp, alpha, beta, gamma, mp,
                                              update_step=(it == 0), step=step)
                es.append(e)
            energies.append(np.array(es))
        return h, hinv, energies

    def max_norm(self, v):
        return float(self.lib.aw_oracle_max_norm(_fp(v[0]), _fp(v[1]), _fp(v[2]),
                                                 ctypes.c_long(v[0].size)))

    # --- greedy iteration -------------------------------------------------------
    def greedy_iterate(self, I0, I1, h, hinv=None, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                       gamma=0.001, max_pert=0.5, update_step=False, step=0.0):
        """One GreedyIteratorCPU::Iterate; h/hinv updated in place.
        Returns (energy, step)."""
        st = ctypes.c_float(step)
        hi = hinv if hinv is not None else [None, None, None]
        e = self.lib.aw_oracle_greedy_iterate(
            _fp(I0), _fp(I1), _fp(h[0]), _fp(h[1]), _fp(h[2]), _fp(hi[0]), _fp(hi[1]),
            _fp(hi[2]), *_shape(I0), *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
            ctypes.c_float(max_pert), _i(int(update_step)), ctypes.byref(st))
        return float(e), float(st.value)

    def ldmm_iterate(self, I0, I1, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001,
                     sigma=0.1, step=0.005, update_step=False, max_pert=0.1, vec=False):
        """One LDMMIteratorCPU::IterateNew; v [T,3,nz,ny,nx] updated in place.
        Returns (image energy sp^3*sum diff^2, step), and with vec the debug
        mode's sum_t <L v_t, v_t> sp^3 of the updated v as a third value."""
        assert v.dtype == np.float32 and v.flags.c_contiguous
        st = ctypes.c_float(step)
        ve = ctypes.c_double(0.0)
        e = self.lib.aw_oracle_ldmm_iterate(_fp(I0), _fp(I1), v.ctypes.data_as(_f), _i(v.shape[0]),
                                            *_shape(I0), *map(_dbl, sp), _dbl(alpha), _dbl(beta),
                                            _dbl(gamma), ctypes.c_float(sigma), ctypes.byref(st),
                                            _i(int(update_step)), ctypes.c_float(max_pert),
                                            ctypes.byref(ve) if vec else None)
        return (float(e), float(st.value)) + ((ve.value,) if vec else ())

    def ldmm_alphas(self, I0, I1, v, sp=(1.0, 1.0, 1.0), sigma=0.1):
        """IterateNew with computeAlphasOnly: alpha_t [T,nz,ny,nx]; returns
        (alphas, image energy)."""
        v = np.ascontiguousarray(v, np.float32)
        T = v.shape[0]
        out = np.empty((T,) + I0.shape, np.float32)
        self.lib.aw_oracle_ldmm_alphas.restype = ctypes.c_double
        e = self.lib.aw_oracle_ldmm_alphas(_fp(I0), _fp(I1), v.ctypes.data_as(_f), _i(T),
                                           *_shape(I0), *map(_dbl, sp), ctypes.c_float(sigma),
                                           out.ctypes.data_as(_f))
        return out, float(e)

    def jacobian(self, v, sp=(1.0, 1.0, 1.0)):
        """|D(x*sp + v)| (HField3DUtils::jacobian of IterateOrig's map)."""
        out = np.empty(v.shape[1:], np.float32)
        self.lib.aw_oracle_jacobian(_fp(v[0]), _fp(v[1]), _fp(v[2]), _fp(out), *_shape(v),
                                    *map(_dbl, sp))
        return out

    def ldmm_iterate_orig(self, I0, I1, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                          gamma=0.001, sigma=0.1, step=0.005, update_step=False, max_pert=0.1,
                          vec=False):
        """One LDMMIteratorCPU::IterateOrig; v updated in place. Returns
        (image energy after the update, step), and with vec the vector energy
        as ldmm_iterate does."""
        assert v.dtype == np.float32 and v.flags.c_contiguous
        st = ctypes.c_float(step)
        ve = ctypes.c_double(0.0)
        e = self.lib.aw_oracle_ldmm_iterate_orig(
            _fp(I0), _fp(I1), v.ctypes.data_as(_f), _i(v.shape[0]), *_shape(I0), *map(_dbl, sp),
            _dbl(alpha), _dbl(beta), _dbl(gamma), ctypes.c_float(sigma), ctypes.byref(st),
            _i(int(update_step)), ctypes.c_float(max_pert), ctypes.byref(ve) if vec else None)
        return (float(e), float(st.value)) + ((ve.value,) if vec else ())

    def ldmm_shoot_iterate(self, I0, I1, alpha0, T, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                           gamma=0.001, sigma=0.1, step=0.005, vec=False):
        """One LDMMShootingIteratorCPU::Iterate; alpha0 [nz,ny,nx] updated in
        place. Returns (image energy, phi0T, phiT0), with vec=True (image
        energy, sum over t of <L v_t, v_t>, phi0T, phiT0)."""
        assert alpha0.dtype == np.float32 and alpha0.flags.c_contiguous
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        ev = ctypes.c_double()
        e = self.lib.aw_oracle_ldmm_shoot_iterate(
            _fp(I0), _fp(I1), _fp(alpha0), p0.ctypes.data_as(_f), p1.ctypes.data_as(_f), _i(T),
            *_shape(I0), *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
            ctypes.c_float(sigma), ctypes.c_float(step), ctypes.byref(ev) if vec else None)
        return (float(e), float(ev.value), p0, p1) if vec else (float(e), p0, p1)

    def ldmm_velshoot_iterate(self, I0, I1, v0, T, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                              gamma=0.001, sigma=0.1, step=0.005, update_step=False,
                              max_pert=0.1):
        """One LDMMVelShootingIteratorCPU::Iterate; v0 [3,nz,ny,nx] updated in
        place (or the step set with update_step). Returns (image energy,
        vector energy, step, phi0T, phiT0)."""
        assert v0.dtype == np.float32 and v0.flags.c_contiguous
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        st = ctypes.c_float(step)
        ev = ctypes.c_double()
        e = self.lib.aw_oracle_ldmm_velshoot_iterate(
            _fp(I0), _fp(I1), _fp(v0), _fp(p0), _fp(p1), _i(T), *_shape(I0), *map(_dbl, sp),
            _dbl(alpha), _dbl(beta), _dbl(gamma), ctypes.c_float(sigma), ctypes.byref(st),
            _i(int(update_step)), ctypes.c_float(max_pert), ctypes.byref(ev))
        return float(e), float(ev.value), float(st.value), p0, p1

    def geodesic_shoot(self, I0, alpha0, T, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                       gamma=0.001):
        """LDMMGeodesicShootingCPU::ShootImage: (phi0T, phiT0, final image)."""
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        img = np.empty(I0.shape, np.float32)
        self.lib.aw_oracle_geodesic_shoot(_fp(I0), _fp(alpha0), _i(T), *_shape(I0), *map(_dbl, sp),
                                          _dbl(alpha), _dbl(beta), _dbl(gamma), _fp(p0), _fp(p1),
                                          _fp(img))
        return p0, p1, img

    def ldmm_adshoot_iterate(self, I0, I1, alpha0, T, sp=(1.0, 1.0, 1.0), alpha=0.01,
                             beta=0.01, gamma=0.001, sigma=0.1, step=0.005):
        """One LDMMAdShootingIteratorCPU::Iterate (shooting, then the backward
        adjoint integration); alpha0 [nz,ny,nx] updated in place. Returns
        (image energy, vector energy <L v0, v0>, V [T,3,...], phi0T, phiT0),
        the maps as the iteration leaves them (at time t_1)."""
        assert alpha0.dtype == np.float32 and alpha0.flags.c_contiguous
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        V = np.empty((T, 3) + I0.shape, np.float32)
        ev = ctypes.c_double()
        e = self.lib.aw_oracle_ldmm_adshoot_iterate(
            _fp(I0), _fp(I1), _fp(alpha0), p0.ctypes.data_as(_f), p1.ctypes.data_as(_f),
            V.ctypes.data_as(_f), _i(T), *_shape(I0), *map(_dbl, sp), _dbl(alpha), _dbl(beta),
            _dbl(gamma), ctypes.c_float(sigma), ctypes.c_float(step), ctypes.byref(ev))
        return float(e), float(ev.value), V, p0, p1

    def adshoot_final_maps(self, V, sp=(1.0, 1.0, 1.0)):
        """finalUpdatePhi0T / finalUpdatePhiT0 (LDMMAdShootingIteratorCPU.cxx:
        433-453): the maps composed from identity through every stored v_t."""
        shape = V.shape[2:]
        p0, p1 = identity(shape), identity(shape)
        for t in range(V.shape[0]):
            p0 = self.compose_vh(V[t], p0, sp, direction=1, bg=BG_PARTIAL_ZERO)
            p1 = self.compose_hv(p1, V[t], sp, direction=-1, bg=BG_PARTIAL_ID)
        return p0, p1

    def resample_image(self, img, new_shape, src_sp, dst_sp):
        """ImageUtils::resampleNew with clamped linear interpolation (the
        MultiscaleManager's image upsampling), origin 0."""
        out = np.empty(new_shape, np.float32)
        mz, my, mx = new_shape
        self.lib.aw_oracle_resample_image(_fp(np.ascontiguousarray(img, np.float32)), *_shape(img),
                                          *map(_dbl, src_sp), _fp(out), _i(mx), _i(my), _i(mz),
                                          *map(_dbl, dst_sp))
        return out

    def adshoot_warp(self, I0, I1, T, levels, sp=(1.0, 1.0, 1.0), sigma=1.0, alpha=0.01,
                     beta=0.01, gamma=0.001):
        """LDMMWarpAd::RunWarp (Algorithms/LDMM/LDMMWarp.txx:72-133,
        LDMMWarpAd.txx:37-42) over levels = [(factor, iters, step)], coarsest
        first after sorting: images Gaussian-downsampled per level, alpha0
        from zero at the first level and resampled (resampleNew) to each next
        one, final maps from the last shooting. Returns (alpha0, phi0T,
        phiT0, [(image energies, vector energies)] per level)."""
        levels = sorted(levels, key=lambda l: -l[0])
        shape = I0.shape
        a0 = None
        prev_sp = None
        V = None
        hist = []
        for li, (f, iters, step) in enumerate(levels):
            size = tuple(n // f for n in shape)
            lsp = tuple(float(np.float32(s) * np.float32(f)) for s in sp)
            if size == tuple(shape):
                a, b = I0, I1
            else:
                a, b = self.downsample(I0, size, sp), self.downsample(I1, size, sp)
            if li == 0:
                a0 = np.zeros(size, np.float32)
            else:
                a0 = self.resample_image(a0, size, prev_sp, lsp)
            prev_sp = lsp
            ei, ev = [], []
            for _ in range(iters):
                e, v, V, _, _ = self.ldmm_adshoot_iterate(a, b, a0, T, lsp, alpha, beta, gamma,
                                                          sigma, step)
                ei.append(e)
                ev.append(v)
            hist.append((np.array(ei), np.array(ev)))
        p0, p1 = self.adshoot_final_maps(V, prev_sp)
        return a0, p0, p1, hist

    def ldmm_i1_at_0(self, I1, v, sp=(1.0, 1.0, 1.0), jacdet=True):
        """LDMMDeformationData::GetI1At0 and LDMMIteratorCPU::ComputeJacDet
        for velocities v [T,3,nz,ny,nx]. Returns (image, JacDet or None)."""
        v = np.ascontiguousarray(v, np.float32)
        img = np.empty(I1.shape, np.float32)
        jd = np.empty(I1.shape, np.float32) if jacdet else None
        self.lib.aw_oracle_ldmm_i1_at_0(_fp(I1), v.ctypes.data_as(_f), _i(v.shape[0]),
                                        *_shape(I1), *map(_dbl, sp), _fp(img),
                                        _fp(jd) if jd is not None else None)
        return img, jd

    def voxel_median(self, imgs, k):
        """MedianCalculator::Select over the images: the per-voxel k-th
        smallest value (0-based) by the reference's bisection. Raises when a
        voxel does not converge, as the reference throws."""
        stack = np.ascontiguousarray(np.stack(imgs), np.float32)
        out = np.empty(imgs[0].shape, np.float32)
        rc = self.lib.aw_oracle_voxel_median(_fp(stack), _i(len(imgs)), ctypes.c_long(out.size),
                                             _i(k), _fp(out))
        if rc == 2:
            raise ValueError("voxel_median: needs images, voxels and 0 <= k < n")
        if rc:
            raise RuntimeError("Select() not converging")
        return out

    @staticmethod
    def median_index(n):
        """LDMMAtlasBuilder::ComputeMedian's index (LDMMAtlasBuilder.txx:222)."""
        return n // 2 - 1 if n % 2 == 0 else n // 2

    def ldmm_atlas_mean_sums(self, imgs, vs, weights, sp=(1.0, 1.0, 1.0), jacobian_scale=True):
        """One node's sums of LDMMAtlasThreadCPU::ComputeThreadMean: (sum w
        I1At0 JacDet, sum w JacDet) with JacobianScale, else (sum w I1At0,
        None); float32, subjects added in order (one thread per image)."""
        acc = np.zeros(imgs[0].shape, np.float32)
        jsum = np.zeros(imgs[0].shape, np.float32) if jacobian_scale else None
        for img, v, w in zip(imgs, vs, weights):
            d, jd = self.ldmm_i1_at_0(img, v, sp, jacdet=jacobian_scale)
            w = np.float32(w)
            if jacobian_scale:
                acc += (d * jd) * w
                jsum += jd * w
            else:
                acc += d * w
        return acc, jsum

    @staticmethod
    def ldmm_distance(img_energy, vec_sum, sigma, T):
        """sqrt(LDMMEnergy::GetEnergy()) as LDMMAtlasThreadCPU::
        FinishImageIteration forms it (LDMMAtlasThreadCPU.cxx:175-181): the
        image term times (1.0/(sigma*sigma)) (LDMMEnergy.h:42) plus the mean
        step energy (LDMMEnergy.cxx:55-64), in float."""
        f = np.float32
        inv = 1.0 / float(f(sigma) * f(sigma))
        e = f(f(inv * float(f(img_energy))) + f(f(vec_sum) / f(T)))
        return f(np.sqrt(e))

    @staticmethod
    def ldmm_atlas_weights(weights, dists, compute_median, trimmed):
        """ComputeThreadMean's per-image weight (LDMMAtlasThreadCPU.cxx:
        221-237) with ComputeMedian (divided by the distance, 1 while it is
        0) and TrimmedMeanSize (LDMMAtlasBuilder::ComputeWeights,
        LDMMAtlasBuilder.txx:437-500: kVal = Select(distances, n, k), the
        images with distance 0 or at most kVal while fewer than k are
        chosen keep their weight, the others 0, then all divided by the sum)."""
        f = np.float32
        w = [f(x) for x in weights]
        if compute_median:
            for i in range(len(w)):
                d = f(dists[i])
                d = f(1.0) if d == 0 else d
                w[i] = f(w[i] * f(1.0 / float(d)))
        if trimmed:
            kval = np.sort(np.asarray(dists, np.float32))[trimmed]
            tw, ws, count = [], f(0.0), 0
            for i in range(len(w)):
                if dists[i] == 0 or (dists[i] <= kval and count < trimmed):
                    tw.append(f(weights[i]))
                    ws = f(ws + f(weights[i]))
                    count += 1
                else:
                    tw.append(f(0.0))
            w = [f(x / ws) for x in tw]
        return w

    def ldmm_atlas_run(self, imgs, weights, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1, step=0.005,
                       adaptive=False, max_pert=0.1, alpha=0.01, beta=0.01, gamma=0.001,
                       use_new=True, jacobian_scale=True, voxel_median=False,
                       compute_median=False, trimmed=0):
        """LDMM relaxation atlas, the AtlasThreadMain loop (Algorithms/Common/
        AtlasThread.txx:97-181) with LDMMAtlasThreadCPU's hooks
        (LDMM/LDMMAtlasThreadCPU.cxx:146-264): mean from v = 0, then per
        iteration every subject's LDMM iteration toward the mean (the
        step-size pass first at iteration 0 when adaptive) and the mean
        again, sum w I1At0 JacDet / sum w JacDet (LDMMAtlasBuilder.txx:
        274-335). Returns (mean, [v_i], image energies [iters, ns])."""
        ns = len(imgs)
        vs = [np.zeros((T, 3) + imgs[0].shape, np.float32) for _ in range(ns)]
        steps = [float(step)] * ns
        it = self.ldmm_iterate if use_new else self.ldmm_iterate_orig
        kw = dict(sp=sp, alpha=alpha, beta=beta, gamma=gamma, sigma=sigma)

        reweigh = compute_median or trimmed > 0
        dists = [np.float32(0.0)] * ns

        def mean_of():
            if voxel_median:  # UsePerVoxelMedian: LDMMAtlasBuilder.txx:336-338
                defs = [self.ldmm_i1_at_0(img, v, sp, jacdet=False)[0]
                        for img, v in zip(imgs, vs)]
                return self.voxel_median(defs, self.median_index(ns))
            w = (self.ldmm_atlas_weights(weights, dists, compute_median, trimmed) if reweigh
                 else weights)
            acc, jsum = self.ldmm_atlas_mean_sums(imgs, vs, w, sp, jacobian_scale)
            return acc / jsum if jacobian_scale else acc

        mean = mean_of()
        en = np.zeros((iters, ns))
        for k in range(iters):
            for i in range(ns):
                if k == 0 and adaptive:
                    _, steps[i] = it(mean, imgs[i], vs[i], step=steps[i], update_step=True,
                                     max_pert=max_pert, **kw)
                r = it(mean, imgs[i], vs[i], step=steps[i], vec=reweigh, **kw)
                en[k, i] = r[0]
                if reweigh:
                    dists[i] = self.ldmm_distance(r[0], r[2], sigma, T)
            mean = mean_of()
        return mean, vs, en

    def ldmm_shoot_atlas_run(self, imgs, weights, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1,
                             step=0.005, alpha=0.01, beta=0.01, gamma=0.001,
                             jacobian_scale=True):
        """The shooting atlas: AtlasThreadMain (Algorithms/Common/AtlasThread.txx:
        97-181) with LDMMShootingAtlasThreadCPU's mean (LDMM/
        LDMMShootingAtlasThreadCPU.cxx:183-224): every subject one
        LDMMShootingIteratorCPU::Iterate toward the mean (I0 = the mean, I1 =
        the subject, LDMMShootingAtlasDefDataCPU, .cxx:42-52), then
        sum w I1(phi0T) J / sum w J with J = forwardApply(ones, phiT0)
        (LDMMShootingIteratorCPU::ComputeJacDet, .cxx:108-119). Returns
        (mean, [alpha0_i], image energies [iters, ns])."""
        ns = len(imgs)
        shape = imgs[0].shape
        a0 = [np.zeros(shape, np.float32) for _ in range(ns)]
        maps = [(identity(shape), identity(shape)) for _ in range(ns)]
        ones = np.ones(shape, np.float32)

        def mean_of():
            acc = np.zeros(shape, np.float32)
            jsum = np.zeros(shape, np.float32)
            for img, (p0, p1), w in zip(imgs, maps, weights):
                d = self.apply(img, p0)
                w = np.float32(w)
                if jacobian_scale:
                    jd = self.splat(ones, p1)
                    acc += (d * jd) * w
                    jsum += jd * w
                else:
                    acc += d * w
            return acc / jsum if jacobian_scale else acc

        mean = mean_of()
        en = np.zeros((iters, ns))
        for k in range(iters):
            for i in range(ns):
                en[k, i], p0, p1 = self.ldmm_shoot_iterate(mean, imgs[i], a0[i], T, sp, alpha,
                                                           beta, gamma, sigma, step)
                maps[i] = (p0, p1)
            mean = mean_of()
        return mean, a0, en

    def greedy_run(self, I0, I1, iters, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001,
                   max_pert=0.5, inverse=False):
        """Single-scale greedy registration from the identity."""
        h = identity(I0.shape)
        hinv = identity(I0.shape) if inverse else None
        energies, step = [], 0.0
        for it in range(iters):
            e, step = self.greedy_iterate(I0, I1, h, hinv, sp, alpha, beta, gamma, max_pert,
                                          update_step=(it == 0), step=step)
            energies.append(e)
        return h, hinv, np.array(energies), step


    # --- atlas ------------------------------------------------------------------
    def apply_atlas(self, img, h):
        """Subject image (own grid) sampled at the atlas map of h (template grid)."""
        out = np.empty(h.shape[1:], np.float32)
        mx, my, mz = _shape(img)
        self.lib.aw_oracle_apply_atlas(_fp(img), _i(mx), _i(my), _i(mz), _fp(h[0]), _fp(h[1]),
                                       _fp(h[2]), _fp(out), *_shape(h))
        return out

    def atlas_mean(self, imgs, hs, weights):
        """GreedyAtlasThreadCPU::ComputeThreadMean over subjects in order."""
        ns = len(imgs)
        shape = hs[0].shape[1:]
        mean = np.empty(shape, np.float32)
        ip = (_f * ns)(*[_fp(a) for a in imgs])
        dims = (ctypes.c_int * (3 * ns))(*[d for a in imgs for d in _shape(a)])
        hp = (_f * (3 * ns))(*[_fp(h[c]) for h in hs for c in range(3)])
        w = (ctypes.c_float * ns)(*weights)
        self.lib.aw_oracle_atlas_mean(ip, dims, hp, w, _i(ns), _fp(mean), *_shape(hs[0]))
        return mean

    def atlas_iterate(self, img, mean, h, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                      gamma=0.001, max_pert=0.5, update_step=False, step=0.0):
        st = ctypes.c_float(step)
        mx, my, mz = _shape(img)
        e = self.lib.aw_oracle_atlas_iterate(
            _fp(img), _i(mx), _i(my), _i(mz), _fp(mean), _fp(h[0]), _fp(h[1]), _fp(h[2]),
            *_shape(h), *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
            ctypes.c_float(max_pert), _i(int(update_step)), ctypes.byref(st))
        return float(e), float(st.value)

    def atlas_run(self, imgs, weights, shape, iters, mean_period=1, sp=(1.0, 1.0, 1.0),
                  alpha=0.01, beta=0.01, gamma=0.001, max_pert=0.5):
        """AtlasThread::AtlasThreadMain at one scale: mean, then per iteration
        one greedy step of every subject toward the mean, the mean recomputed
        after every mean_period-th iteration. Returns (mean, [h_i],
        energies [iters, ns], steps)."""
        hs = [identity(shape) for _ in imgs]
        mean = self.atlas_mean(imgs, hs, weights)
        steps = [0.0] * len(imgs)
        en = np.zeros((iters, len(imgs)))
        for it in range(iters):
            for k, img in enumerate(imgs):
                en[it, k], steps[k] = self.atlas_iterate(img, mean, hs[k], sp, alpha, beta, gamma,
                                                         max_pert, it == 0, steps[k])
            if (it + 1) % mean_period == 0:
                mean = self.atlas_mean(imgs, hs, weights)
        return mean, hs, en, steps


_quiet_lock = threading.Lock()
_quiet_depth = 0
_quiet_saved = None


@contextlib.contextmanager
def quiet_stdout():
    """Send fd 1 to /dev/null while the reference code runs: its parameter
    parser prints diagnostics on std::cout. Re-entrant across threads."""
    global _quiet_depth, _quiet_saved
    with _quiet_lock:
        if _quiet_depth == 0:
            sys.stdout.flush()
            _quiet_saved = os.dup(1)
            devnull = os.open(os.devnull, os.O_WRONLY)
            os.dup2(devnull, 1)
            os.close(devnull)
        _quiet_depth += 1
    try:
        yield
    finally:
        with _quiet_lock:
            _quiet_depth -= 1
            if _quiet_depth == 0:
                libc = ctypes.CDLL(None)
                libc.fflush(None)
                os.dup2(_quiet_saved, 1)
                os.close(_quiet_saved)
                _quiet_saved = None


class Reference:
    """ctypes wrapper of the reference's own CPU code (oracle/_ref/libawref.so)."""

    def __init__(self, path: str = REF_SO):
        self.lib = ctypes.CDLL(path)
        self.lib.awref_last_error.restype = ctypes.c_char_p

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.awref_last_error().decode())

    def apply(self, img, h):
        out = np.empty_like(img)
        self._check(self.lib.awref_apply(_fp(img), _fp(h[0]), _fp(h[1]), _fp(h[2]), _fp(out),
                                         *_shape(img)))
        return out

    def gradient(self, img, sp=(1.0, 1.0, 1.0), wrap=False):
        g = np.zeros((3,) + img.shape, np.float32)
        self._check(self.lib.awref_gradient(_fp(img), _fp(g[0]), _fp(g[1]), _fp(g[2]),
                                            *_shape(img), *map(_dbl, sp), _i(int(wrap))))
        return g

    def compose_hv(self, g, v, sp=(1.0, 1.0, 1.0), direction=1, bg=BG_PARTIAL_ID):
        o = np.empty_like(g)
        self._check(self.lib.awref_compose_hv(_fp(g[0]), _fp(g[1]), _fp(g[2]), _fp(v[0]),
                                              _fp(v[1]), _fp(v[2]), _fp(o[0]), _fp(o[1]),
                                              _fp(o[2]), *_shape(g), *map(_dbl, sp),
                                              _i(direction), _i(bg)))
        return o

    def compose_vh(self, v, g, sp=(1.0, 1.0, 1.0), direction=-1, bg=BG_PARTIAL_ZERO):
        o = np.empty_like(g)
        self._check(self.lib.awref_compose_vh(_fp(v[0]), _fp(v[1]), _fp(v[2]), _fp(g[0]),
                                              _fp(g[1]), _fp(g[2]), _fp(o[0]), _fp(o[1]),
                                              _fp(o[2]), *_shape(g), *map(_dbl, sp),
                                              _i(direction), _i(bg)))
        return o

    def splat(self, img, h):
        out = np.empty_like(img)
        self._check(self.lib.awref_splat(_fp(img), _fp(h[0]), _fp(h[1]), _fp(h[2]), _fp(out),
                                         *_shape(img)))
        return out

    def downsample(self, img, new_shape, sp=(1.0, 1.0, 1.0)):
        out = np.empty(new_shape, np.float32)
        mz, my, mx = new_shape
        with quiet_stdout():
            rc = self.lib.awref_downsample(_fp(img), *_shape(img), *map(_dbl, sp), _fp(out),
                                           _i(mx), _i(my), _i(mz))
        self._check(rc)
        return out

    def upsample_hfield(self, h, new_shape, rescale=True):
        out = np.empty((3,) + tuple(new_shape), np.float32)
        mz, my, mx = new_shape
        self._check(self.lib.awref_upsample_hfield(_fp(np.ascontiguousarray(h)), *_shape(h),
                                                   _fp(out), _i(mx), _i(my), _i(mz),
                                                   _i(int(rescale))))
        return out

    def fluid(self, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001, inverse=True):
        o = np.ascontiguousarray(v, dtype=np.float32).copy()
        self._check(self.lib.awref_fluid(_fp(o[0]), _fp(o[1]), _fp(o[2]), *_shape(o),
                                         *map(_dbl, sp), _dbl(alpha), _dbl(beta), _dbl(gamma),
                                         _i(int(inverse))))
        return o

    def fluid_f64(self, v, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001, inverse=True):
        o = np.ascontiguousarray(v, dtype=np.float64).copy()
        self._check(self.lib.awref_fluid_f64(_dp(o[0]), _dp(o[1]), _dp(o[2]), *_shape(o),
                                             *map(_dbl, sp), _dbl(alpha), _dbl(beta),
                                             _dbl(gamma), _i(int(inverse))))
        return o

    def greedy_open(self, I0, I1, max_pert=0.5, alpha=0.01, beta=0.01, gamma=0.001,
                    inverse=False):
        """A single-scale GreedyIteratorCPU registration kept open (unit
        spacing): builds the data object, iterator and FFT plans and runs
        iteration 0 (the step update). Returns a handle for greedy_iterate."""
        self.lib.awref_greedy_open.restype = ctypes.c_void_p
        with quiet_stdout():
            h = self.lib.awref_greedy_open(_fp(I0), _fp(I1), *_shape(I0), ctypes.c_float(max_pert),
                                           _dbl(alpha), _dbl(beta), _dbl(gamma), _i(int(inverse)))
        if not h:
            raise RuntimeError(self.lib.awref_last_error().decode())
        return ctypes.c_void_p(h)

    def greedy_iterate(self, handle, n_iters=1) -> float:
        """n_iters further GreedyIteratorCPU::Iterate calls; returns the last energy."""
        e = ctypes.c_double()
        self._check(self.lib.awref_greedy_iterate(handle, _i(n_iters), ctypes.byref(e)))
        return float(e.value)

    def greedy_close(self, handle):
        self.lib.awref_greedy_close(handle)

    def greedy_run(self, I0, I1, factors: Sequence[int], iters: Sequence[int],
                   max_pert: Sequence[float], sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                   gamma=0.001, inverse=False, h_init=None, hinv_init=None, init_step=0.0,
                   skip_step_update=False):
        """GreedyIteratorCPU driven through the GreedyWarp::RunWarp scale loop."""
        ns = len(factors)
        fa = (ctypes.c_int * ns)(*factors)
        it = (ctypes.c_int * ns)(*iters)
        mp = (ctypes.c_float * ns)(*max_pert)
        h = np.empty((3,) + I0.shape, np.float32)
        hinv = np.empty((3,) + I0.shape, np.float32) if inverse else None
        total = int(sum(iters))
        en = np.zeros(total, np.float64)
        steps = np.zeros(total, np.float32)
        hi = np.ascontiguousarray(h_init, np.float32) if h_init is not None else None
        hii = np.ascontiguousarray(hinv_init, np.float32) if hinv_init is not None else None
        with quiet_stdout():
            rc = self.lib.awref_greedy_run(
            _fp(I0), _fp(I1), *_shape(I0), *map(_dbl, sp), _i(ns), fa, it, mp, _dbl(alpha),
            _dbl(beta), _dbl(gamma), _i(int(inverse)), _fp(hi), _fp(hii),
            ctypes.c_float(init_step), _i(int(skip_step_update)), _fp(h), _fp(hinv), _dp(en),
            _fp(steps))
        self._check(rc)
        return h, hinv, en, steps

    def ldmm_run(self, I0, I1, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1, step=0.005,
                 adaptive=False, max_pert=0.1, alpha=0.01, beta=0.01, gamma=0.001,
                 use_new=True, debug=True, v_init=None, vec_out=None):
        """LDMMIteratorCPU (IterateNew when use_new) through the LDMMWarp loop
        at one scale. Returns (v [T,3,...], image energies, step)."""
        n = I0.size
        v = (np.ascontiguousarray(v_init, np.float32).copy() if v_init is not None
             else np.zeros((T, 3) + I0.shape, np.float32))
        en = np.zeros(iters, np.float64)
        st = ctypes.c_float()
        with quiet_stdout():
            rc = self.lib.awref_ldmm_run(
                _fp(I0), _fp(I1), *_shape(I0), *map(_dbl, sp), _i(T), _i(iters),
                ctypes.c_float(sigma), ctypes.c_float(step), _i(int(adaptive)),
                ctypes.c_float(max_pert), _dbl(alpha), _dbl(beta), _dbl(gamma), _i(int(use_new)),
                _i(int(debug)), _i(int(v_init is not None)), v.ctypes.data_as(_f), _dp(en),
                ctypes.byref(st), _dp(vec_out) if vec_out is not None else None)
        self._check(rc)
        return v, en, float(st.value)

    def ldmm_i1_at_0(self, I1, v, sp=(1.0, 1.0, 1.0)):
        """The reference's GetI1At0 and ComputeJacDet for velocities v."""
        v = np.ascontiguousarray(v, np.float32)
        img = np.empty(I1.shape, np.float32)
        jd = np.empty(I1.shape, np.float32)
        with quiet_stdout():
            rc = self.lib.awref_ldmm_i1_at_0(_fp(I1), v.ctypes.data_as(_f), *_shape(I1),
                                             *map(_dbl, sp), _i(v.shape[0]), _fp(img), _fp(jd))
        self._check(rc)
        return img, jd

    def shoot_run(self, I0, I1, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1, step=0.005, alpha=0.01,
                  beta=0.01, gamma=0.001, vec=False):
        """The reference's LDMMShootingDefData / LDMMShootingIteratorCPU for
        `iters` iterations from alpha0 = 0. Returns (alpha0, phi0T, phiT0,
        image energies), with vec=True also the per-iteration sums over t of
        the step energies <L v_t, v_t>."""
        a0 = np.empty(I0.shape, np.float32)
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        en = np.zeros(iters, np.float64)
        ev = np.zeros(iters, np.float64)
        with quiet_stdout():
            rc = self.lib.awref_shoot_run(
                _fp(I0), _fp(I1), *_shape(I0), *map(_dbl, sp), _i(T), _i(iters),
                ctypes.c_float(sigma), ctypes.c_float(step), _dbl(alpha), _dbl(beta), _dbl(gamma),
                _fp(a0), p0.ctypes.data_as(_f), p1.ctypes.data_as(_f), _dp(en), _dp(ev))
        self._check(rc)
        return (a0, p0, p1, en, ev) if vec else (a0, p0, p1, en)

    def velshoot_run(self, I0, I1, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1, step=0.005,
                     adaptive=False, max_pert=0.1, alpha=0.01, beta=0.01, gamma=0.001):
        """The reference's LDMMVelShootingIteratorCPU through the LDMMWarp loop
        at one scale. Returns (v0, phi0T, phiT0, image energies, vector
        energies, step)."""
        v0 = np.empty((3,) + I0.shape, np.float32)
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        en = np.zeros(iters, np.float64)
        ve = np.zeros(iters, np.float64)
        st = ctypes.c_float()
        with quiet_stdout():
            rc = self.lib.awref_velshoot_run(
                _fp(I0), _fp(I1), *_shape(I0), *map(_dbl, sp), _i(T), _i(iters),
                ctypes.c_float(sigma), ctypes.c_float(step), _i(int(adaptive)),
                ctypes.c_float(max_pert), _dbl(alpha), _dbl(beta), _dbl(gamma), _fp(v0), _fp(p0),
                _fp(p1), _dp(en), _dp(ve), ctypes.byref(st))
        self._check(rc)
        return v0, p0, p1, en, ve, float(st.value)

    def geodesic_shoot(self, I0, alpha0, T, sp=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01,
                       gamma=0.001):
        """The reference's LDMMGeodesicShootingCPU::ShootImage."""
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        img = np.empty(I0.shape, np.float32)
        with quiet_stdout():
            rc = self.lib.awref_geodesic_shoot(_fp(I0), _fp(alpha0), *_shape(I0), *map(_dbl, sp),
                                               _i(T), _dbl(alpha), _dbl(beta), _dbl(gamma),
                                               _fp(p0), _fp(p1), _fp(img))
        self._check(rc)
        return p0, p1, img

    def adshoot_run(self, I0, I1, T, levels, sp=(1.0, 1.0, 1.0), sigma=1.0, alpha=0.01,
                    beta=0.01, gamma=0.001):
        """The reference's LDMMShootingDefData / LDMMAdShootingIteratorCPU
        through the LDMMWarpAd scale loop; levels = [(factor, iters, step)]
        in parameter-file order. Returns (alpha0, phi0T, phiT0, image
        energies, vector energies), the maps from FinishWarp."""
        ns = len(levels)
        fa = (ctypes.c_int * ns)(*[l[0] for l in levels])
        it = (ctypes.c_int * ns)(*[l[1] for l in levels])
        st = (ctypes.c_float * ns)(*[l[2] for l in levels])
        a0 = np.empty(I0.shape, np.float32)
        p0 = np.empty((3,) + I0.shape, np.float32)
        p1 = np.empty((3,) + I0.shape, np.float32)
        total = int(sum(l[1] for l in levels))
        ei = np.zeros(total, np.float64)
        ev = np.zeros(total, np.float64)
        with quiet_stdout():
            rc = self.lib.awref_adshoot_run(
                _fp(I0), _fp(I1), *_shape(I0), *map(_dbl, sp), _i(T), _i(ns), fa, it, st,
                ctypes.c_float(sigma), _dbl(alpha), _dbl(beta), _dbl(gamma), _fp(a0),
                p0.ctypes.data_as(_f), p1.ctypes.data_as(_f), _dp(ei), _dp(ev))
        self._check(rc)
        return a0, p0, p1, ei, ev

    def voxel_median(self, imgs, k):
        """The reference's MedianCalculator::Select over the images."""
        stack = np.ascontiguousarray(np.stack(imgs), np.float32)
        out = np.empty(imgs[0].shape, np.float32)
        with quiet_stdout():
            rc = self.lib.awref_voxel_median(_fp(stack), _i(len(imgs)), *_shape(imgs[0]), _i(k),
                                             _fp(out))
        if rc == 1:
            raise RuntimeError("Select() not converging")
        self._check(rc)
        return out

    def ldmm_atlas_run(self, imgs, weights, T, iters, sp=(1.0, 1.0, 1.0), sigma=0.1, step=0.005,
                       adaptive=False, max_pert=0.1, alpha=0.01, beta=0.01, gamma=0.001,
                       use_new=True, jacobian_scale=True):
        """The reference's LDMMDeformationData / LDMMIteratorCPU driven through
        the AtlasThreadMain loop with the LDMM atlas thread's mean. Returns
        (mean, [v_i], image energies [iters, ns])."""
        ns = len(imgs)
        n = imgs[0].size
        stack = np.ascontiguousarray(np.stack(imgs), np.float32)
        w = (ctypes.c_float * ns)(*weights)
        mean = np.empty(imgs[0].shape, np.float32)
        v = np.zeros((ns, T, 3) + imgs[0].shape, np.float32)
        en = np.zeros((iters, ns), np.float64)
        with quiet_stdout():
            rc = self.lib.awref_ldmm_atlas_run(
                stack.ctypes.data_as(_f), _i(ns), w, *_shape(imgs[0]), *map(_dbl, sp), _i(T),
                _i(iters), ctypes.c_float(sigma), ctypes.c_float(step), _i(int(adaptive)),
                ctypes.c_float(max_pert), _dbl(alpha), _dbl(beta), _dbl(gamma), _i(int(use_new)),
                _i(int(jacobian_scale)), _fp(mean), v.ctypes.data_as(_f), _dp(en))
        self._check(rc)
        return mean, [v[k] for k in range(ns)], en

    def atlas_run(self, imgs, weights, iters, mean_period=1, sp=(1.0, 1.0, 1.0), alpha=0.01,
                  beta=0.01, gamma=0.001, max_pert=0.5):
        """The reference's GreedyDeformationData / GreedyIteratorCPU driven
        through the AtlasThreadMain loop (equal grids). Returns (mean, [h_i],
        energies [iters, ns])."""
        ns = len(imgs)
        shape = imgs[0].shape
        n = imgs[0].size
        stack = np.ascontiguousarray(np.stack(imgs), np.float32)
        w = (ctypes.c_float * ns)(*weights)
        mean = np.empty(shape, np.float32)
        h = np.empty((ns, 3) + shape, np.float32)
        en = np.zeros((iters, ns), np.float64)
        with quiet_stdout():
            rc = self.lib.awref_atlas_run(
                stack.ctypes.data_as(_f), _i(ns), w, *_shape(imgs[0]), *map(_dbl, sp), _i(iters),
                ctypes.c_float(max_pert), _dbl(alpha), _dbl(beta), _dbl(gamma), _i(mean_period),
                _fp(mean), h.ctypes.data_as(_f), _dp(en))
        self._check(rc)
        return mean, [h[k] for k in range(ns)], en
