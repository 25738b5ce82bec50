/*
 * aw_ref_harness.cxx — C entry points over the reference's own CPU code,
 * compiled from the reference sources (recipe: oracle/ref/Makefile) into
 * oracle/_ref/libawref.so.
 *
 * TEST INFRASTRUCTURE: used to pin the oracle (oracle/aw_oracle.c) against
 * the reference itself and, in bench.py's reference arm, as the timed CPU
 * baseline. The harness only converts planar float arrays to the
 * reference's Array3D<Vector3D<float>> / Image<float> types and calls the
 * reference routines; the drivers below repeat the steps of
 * GreedyWarp::RunWarp (Algorithms/Greedy/GreedyWarp.txx:71-125) and
 * LDMMWarp::RunWarp (Algorithms/LDMM/LDMMWarp.txx:71-130) without their
 * ITK file output.
 */
#include <cstdio>
#include <cstring>
#include <exception>
#include <sstream>
#include <string>
#include <vector>

#include "DiffOper.h"
#include "GreedyDeformationData.h"
#include "GreedyIteratorCPU.h"
#include "GreedyParam.h"
#include "HField3DUtils.h"
#include "ImageUtils.h"
#include "LDMMAdShootingIteratorCPU.h"
#include "LDMMDeformationData.h"
#include "LDMMEnergy.h"
#include "LDMMGeodesicShootingCPU.h"
#include "LDMMIteratorCPU.h"
#include "LDMMParam.h"
#include "LDMMShootingDefData.h"
#include "LDMMShootingIteratorCPU.h"
#include "LDMMVelShootingDefData.h"
#include "LDMMVelShootingIteratorCPU.h"
#include "MedianCalculator.h"
#include "MultiscaleManager.h"
#include "tinyxml.h"

namespace {

std::string g_err;

void to_vf(const float *x, const float *y, const float *z, VectorField &vf) {
  const unsigned n = vf.getNumElements();
  for (unsigned i = 0; i < n; ++i) {
    vf(i).x = x[i];
    vf(i).y = y[i];
    vf(i).z = z[i];
  }
}

void from_vf(const VectorField &vf, float *x, float *y, float *z) {
  const unsigned n = vf.getNumElements();
  for (unsigned i = 0; i < n; ++i) {
    x[i] = vf(i).x;
    y[i] = vf(i).y;
    z[i] = vf(i).z;
  }
}

void to_im(const float *a, Array3D<float> &im) {
  std::memcpy(im.getDataPointer(), a, sizeof(float) * im.getNumElements());
}

void from_im(const Array3D<float> &im, float *a) {
  std::memcpy(a, im.getDataPointer(), sizeof(float) * im.getNumElements());
}

HField3DUtils::VectorBackgroundStrategy bg_of(int b) {
  return static_cast<HField3DUtils::VectorBackgroundStrategy>(b);
}

std::string diffoper_xml(double alpha, double beta, double gamma) {
  std::ostringstream s;
  s.precision(17);
  s << "<DiffOper><Alpha val=\"" << alpha << "\"/><Beta val=\"" << beta << "\"/><Gamma val=\""
    << gamma << "\"/><UseEigenLUT val=\"false\"/><DivergenceFree val=\"false\"/>"
    << "<FFTWNumberOfThreads val=\"1\"/><FFTWMeasure val=\"false\"/></DiffOper>";
  return s.str();
}

template <class P>
void parse_into(P &param, const std::string &xml) {
  TiXmlDocument doc;
  doc.Parse(xml.c_str());
  if (doc.Error()) throw std::runtime_error(std::string("param xml: ") + doc.ErrorDesc());
  param.Parse(doc.RootElement());
}

#define GUARD_BEGIN try {
#define GUARD_END                          \
  }                                        \
  catch (const std::exception &e) {        \
    g_err = e.what();                      \
    return -1;                             \
  }                                        \
  catch (...) {                            \
    g_err = "unknown exception";           \
    return -1;                             \
  }                                        \
  return 0;

// LDMMIteratorCPU with the splatting gradient (IterateNew) selected: the
// reference keeps the selector protected (LDMM/LDMMIteratorCPU.cxx:33,
// LDMMIteratorCPU.h:115), so a subclass sets it before SetScaleLevel.
class LDMMIteratorNewCPU : public LDMMIteratorCPU {
 public:
  LDMMIteratorNewCPU(const SizeType &size, const OriginType &origin, const SpacingType &spacing,
                     unsigned int nTimeSteps, bool debug, bool use_new)
      : LDMMIteratorCPU(size, origin, spacing, nTimeSteps, debug) {
    mUseOrigGradientCalc = !use_new;
  }
};

}  // namespace

extern "C" {

const char *awref_last_error() { return g_err.c_str(); }

/* HField3DUtils::apply, default (zero) background */
int awref_apply(const float *img, const float *hx, const float *hy, const float *hz, float *out,
                int nx, int ny, int nz) {
  GUARD_BEGIN
  Array3D<float> I(nx, ny, nz), O(nx, ny, nz);
  VectorField h(nx, ny, nz);
  to_im(img, I);
  to_vf(hx, hy, hz, h);
  HField3DUtils::apply(I, h, O);
  from_im(O, out);
  GUARD_END
}

/* Array3DUtils::computeGradient */
int awref_gradient(const float *img, float *gx, float *gy, float *gz, int nx, int ny, int nz,
                   double spx, double spy, double spz, int wrap) {
  GUARD_BEGIN
  Array3D<float> I(nx, ny, nz);
  VectorField g(nx, ny, nz);
  to_im(img, I);
  Array3DUtils::computeGradient(I, g, Vector3D<double>(spx, spy, spz), wrap != 0);
  from_vf(g, gx, gy, gz);
  GUARD_END
}

/* composeHV (dir=+1) / composeHVInv (dir=-1): h(x) = g(x +- v(x)/sp) */
int awref_compose_hv(const float *gx, const float *gy, const float *gz, const float *vx,
                     const float *vy, const float *vz, float *ox, float *oy, float *oz, int nx,
                     int ny, int nz, double spx, double spy, double spz, int dir, int bgs) {
  GUARD_BEGIN
  VectorField g(nx, ny, nz), v(nx, ny, nz), h(nx, ny, nz);
  to_vf(gx, gy, gz, g);
  to_vf(vx, vy, vz, v);
  Vector3D<double> sp(spx, spy, spz);
  if (dir > 0)
    HField3DUtils::composeHV(g, v, h, sp, bg_of(bgs));
  else
    HField3DUtils::composeHVInv(g, v, h, sp, bg_of(bgs));
  from_vf(h, ox, oy, oz);
  GUARD_END
}

/* composeVH (dir=+1) / composeVHInv (dir=-1): h(x) = g(x) +- v(g(x))/sp */
int awref_compose_vh(const float *vx, const float *vy, const float *vz, const float *gx,
                     const float *gy, const float *gz, float *ox, float *oy, float *oz, int nx,
                     int ny, int nz, double spx, double spy, double spz, int dir, int bgs) {
  GUARD_BEGIN
  VectorField g(nx, ny, nz), v(nx, ny, nz), h(nx, ny, nz);
  to_vf(gx, gy, gz, g);
  to_vf(vx, vy, vz, v);
  Vector3D<double> sp(spx, spy, spz);
  if (dir > 0)
    HField3DUtils::composeVH(v, g, h, sp, bg_of(bgs));
  else
    HField3DUtils::composeVHInv(v, g, h, sp, bg_of(bgs));
  from_vf(h, ox, oy, oz);
  GUARD_END
}

/* HField3DUtils::forwardApply(image, h, out, 0, false): splatting */
int awref_splat(const float *img, const float *hx, const float *hy, const float *hz, float *out,
                int nx, int ny, int nz) {
  GUARD_BEGIN
  Array3D<float> I(nx, ny, nz), O(nx, ny, nz);
  VectorField h(nx, ny, nz);
  to_im(img, I);
  to_vf(hx, hy, hz, h);
  HField3DUtils::forwardApply(I, h, O, 0.0f, false);
  from_im(O, out);
  GUARD_END
}

/* DiffOperT<float>: L (inverse=0) or L^-1 (inverse=1), in place */
int awref_fluid(float *vx, float *vy, float *vz, int nx, int ny, int nz, double spx, double spy,
                double spz, double alpha, double beta, double gamma, int inverse) {
  GUARD_BEGIN
  DiffOperParam param;
  parse_into(param, diffoper_xml(alpha, beta, gamma));
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  DiffOperT<float> op(size, sp, param);
  VectorField v(nx, ny, nz);
  to_vf(vx, vy, vz, v);
  op.CopyIn(v);
  if (inverse)
    op.ApplyInverseOperator();
  else
    op.ApplyOperator();
  op.CopyOut(v);
  from_vf(v, vx, vy, vz);
  GUARD_END
}

/* DiffOperT<double>: the same operator in FP64 (DiffOper.cxx:1221) */
int awref_fluid_f64(double *vx, double *vy, double *vz, int nx, int ny, int nz, double spx,
                    double spy, double spz, double alpha, double beta, double gamma, int inverse) {
  GUARD_BEGIN
  DiffOperParam param;
  parse_into(param, diffoper_xml(alpha, beta, gamma));
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  DiffOperT<double> op(size, sp, param);
  typename DiffOperT<double>::FFTWVectorField *f = op.GetInternalFFTWVectorField();
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = ((long)z * ny + y) * nx + x;
        (*f)(x, y, z) = Vector3D<double>(vx[i], vy[i], vz[i]);
      }
  if (inverse)
    op.ApplyInverseOperator();
  else
    op.ApplyOperator();
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = ((long)z * ny + y) * nx + x;
        vx[i] = (*f)(x, y, z).x;
        vy[i] = (*f)(x, y, z).y;
        vz[i] = (*f)(x, y, z).z;
      }
  GUARD_END
}

/*
 * Greedy registration through GreedyIteratorCPU, scale loop of
 * GreedyWarp::RunWarp. factors[s] / iters[s] / maxpert[s] per scale level,
 * listed coarse to fine. h (and hinv when compute_inverse) are returned at
 * full resolution; energies[] receives one value per Iterate call.
 * If h_init is non-NULL it replaces the identity initial deformation at the
 * first (and only) scale, with init_step as the starting step size and the
 * step-size update at iteration 0 skipped when skip_step_update is set —
 * this lets a test run single iterations from any state.
 */
int awref_greedy_run(const float *i0, const float *i1, int nx, int ny, int nz, double spx,
                     double spy, double spz, int nscales, const int *factors, const int *iters,
                     const float *maxpert, double alpha, double beta, double gamma,
                     int compute_inverse, const float *h_init, const float *hinv_init,
                     float init_step, int skip_step_update, float *h_out, float *hinv_out,
                     double *energies, float *steps_out) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<GreedyWarpParameterFile>";
  for (int s = 0; s < nscales; ++s) {
    xml << "<GreedyScaleLevel><ScaleLevel><DownsampleFactor val=\"" << factors[s]
        << "\"/></ScaleLevel><GreedyIterator>" << diffoper_xml(alpha, beta, gamma)
        << "<MaxPert val=\"" << maxpert[s] << "\"/></GreedyIterator><NIterations val=\""
        << iters[s] << "\"/></GreedyScaleLevel>";
  }
  xml << "<AutoStepReduce val=\"false\"/></GreedyWarpParameterFile>";
  GreedyParam param;
  parse_into(param, xml.str());

  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i0, I0);
  to_im(i1, I1);

  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(true);
  GreedyDeformationData data(&I0, &I1, param);
  data.ComputeInverseHField(compute_inverse != 0);
  GreedyIteratorCPU iterator(size, origin, sp, true);
  const unsigned nlev = param.GetNumberOfScaleLevels();
  int e = 0;
  data.InitializeWarp();
  for (unsigned level = 0; level < nlev; ++level) {
    scaleManager.SetScaleLevel(level);
    iterator.SetScaleLevel(scaleManager, param.GetScaleLevel(level).Iterator());
    data.SetScaleLevel(scaleManager);
    if (h_init && level == 0) {
      to_vf(h_init, h_init + (long)nx * ny * nz, h_init + 2L * nx * ny * nz, data.Def1To0());
      if (compute_inverse && hinv_init)
        to_vf(hinv_init, hinv_init + (long)nx * ny * nz, hinv_init + 2L * nx * ny * nz,
              data.Def0To1());
      data.StepSize(init_step);
    }
    const unsigned nIters = param.GetScaleLevel(level).NIterations();
    for (unsigned iter = 0; iter < nIters; ++iter) {
      data.SetCurIter(iter);
      if (iter == 0 && !(h_init && skip_step_update)) iterator.UpdateStepSizeNextIteration();
      iterator.Iterate(data);
      if (energies) energies[e] = data.GetEnergyHistory().LastEnergy()->GetEnergy();
      if (steps_out) steps_out[e] = data.StepSize();
      ++e;
    }
  }
  const long n = (long)nx * ny * nz;
  from_vf(data.Def1To0(), h_out, h_out + n, h_out + 2 * n);
  if (compute_inverse && hinv_out) from_vf(data.Def0To1(), hinv_out, hinv_out + n, hinv_out + 2 * n);
  GUARD_END
}

/* A single-scale greedy registration kept open across calls, so a caller can
 * time steady-state GreedyIteratorCPU::Iterate calls on one data object,
 * iterator, DiffOper and FFT plan: awref_greedy_open builds them and runs
 * iteration 0 (the step-size update of GreedyWarp.txx:99), awref_greedy_iterate
 * runs further iterations at that step, awref_greedy_close frees it all. */
struct AwRefGreedy {
  GreedyParam param;
  RealImage I0, I1;
  MultiscaleManager *sm = nullptr;
  GreedyDeformationData *data = nullptr;
  GreedyIteratorCPU *it = nullptr;
  unsigned iter = 0;
  AwRefGreedy(const SizeType &size, const OriginType &o, const SpacingType &sp)
      : I0(size, o, sp), I1(size, o, sp) {}
  ~AwRefGreedy() {
    delete it;
    delete data;
    delete sm;
  }
};

void *awref_greedy_open(const float *i0, const float *i1, int nx, int ny, int nz, float maxpert,
                        double alpha, double beta, double gamma, int compute_inverse) {
  AwRefGreedy *g = nullptr;
  try {
    std::ostringstream xml;
    xml.precision(17);
    xml << "<GreedyWarpParameterFile><GreedyScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
        << "</ScaleLevel><GreedyIterator>" << diffoper_xml(alpha, beta, gamma)
        << "<MaxPert val=\"" << maxpert << "\"/></GreedyIterator><NIterations val=\"1000000\"/>"
        << "</GreedyScaleLevel><AutoStepReduce val=\"false\"/></GreedyWarpParameterFile>";
    SizeType size(nx, ny, nz);
    SpacingType sp(1.0, 1.0, 1.0);
    OriginType origin(0, 0, 0);
    g = new AwRefGreedy(size, origin, sp);
    parse_into(g->param, xml.str());
    to_im(i0, g->I0);
    to_im(i1, g->I1);
    g->sm = new MultiscaleManager(size, sp, origin, g->param);
    g->sm->SetScaleVectorFields(true);
    g->data = new GreedyDeformationData(&g->I0, &g->I1, g->param);
    g->data->ComputeInverseHField(compute_inverse != 0);
    g->it = new GreedyIteratorCPU(size, origin, sp, true);
    g->data->InitializeWarp();
    g->sm->SetScaleLevel(0);
    g->it->SetScaleLevel(*g->sm, g->param.GetScaleLevel(0).Iterator());
    g->data->SetScaleLevel(*g->sm);
    g->data->SetCurIter(0);
    g->it->UpdateStepSizeNextIteration();
    g->it->Iterate(*g->data);
    g->iter = 1;
    return g;
  } catch (const std::exception &e) {
    g_err = e.what();
  } catch (...) {
    g_err = "unknown exception";
  }
  delete g;
  return nullptr;
}

int awref_greedy_iterate(void *handle, int n_iters, double *last_energy) {
  GUARD_BEGIN
  AwRefGreedy *g = static_cast<AwRefGreedy *>(handle);
  for (int k = 0; k < n_iters; ++k) {
    g->data->SetCurIter(g->iter++);
    g->it->Iterate(*g->data);
  }
  if (last_energy) *last_energy = g->data->GetEnergyHistory().LastEnergy()->GetEnergy();
  GUARD_END
}

void awref_greedy_close(void *handle) { delete static_cast<AwRefGreedy *>(handle); }

/* Greedy atlas on one node and one thread, one scale, equal grids: the loop
 * of AtlasThread::AtlasThreadMain (Algorithms/Common/AtlasThread.txx:97-181)
 * over the reference's GreedyDeformationData with I1 = the shared mean and
 * ScaleI1 off (the set-up of GreedyAtlasDefDataCPU), one GreedyIteratorCPU
 * for all subjects (Greedy/GreedyAtlasThreadCPU.cxx InitThread), the step
 * recomputed at iteration 0 (BeginImageIteration), and the mean of
 * GreedyAtlasThreadCPU::ComputeThreadMean via GetI0At1, recomputed after
 * every `mean_period`-th iteration (1: after every iteration, as there).
 * imgs: ns images back to back; h_out: ns x 3 planes; energies: iters x ns. */
int awref_atlas_run(const float *imgs, int ns, const float *weights, int nx, int ny, int nz,
                    double spx, double spy, double spz, int iters, float maxpert, double alpha,
                    double beta, double gamma, int mean_period, float *mean_out, float *h_out,
                    double *energies) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<GreedyWarpParameterFile><GreedyScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><GreedyIterator>" << diffoper_xml(alpha, beta, gamma)
      << "<MaxPert val=\"" << maxpert << "\"/></GreedyIterator><NIterations val=\"" << iters
      << "\"/></GreedyScaleLevel><AutoStepReduce val=\"false\"/></GreedyWarpParameterFile>";
  GreedyParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  const long n = (long)nx * ny * nz;
  RealImage mean(size, origin, sp);
  mean.fill(0.f);
  std::vector<RealImage *> ims;
  std::vector<GreedyDeformationData *> data;
  for (int i = 0; i < ns; ++i) {
    ims.push_back(new RealImage(size, origin, sp));
    to_im(imgs + i * n, *ims.back());
    data.push_back(new GreedyDeformationData(ims.back(), &mean, param));
    data.back()->ScaleI1(false);
  }
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(true);
  GreedyIteratorCPU iterator(size, origin, sp, true);
  for (auto *d : data) d->InitializeWarp();
  scaleManager.SetScaleLevel(0);
  iterator.SetScaleLevel(scaleManager, param.GetScaleLevel(0).Iterator());
  for (auto *d : data) d->SetScaleLevel(scaleManager);
  RealImage defIm(size, origin, sp);
  auto thread_mean = [&]() {
    mean.fill(0.0);
    Real *avg = mean.getDataPointer();
    for (int i = 0; i < ns; ++i) {
      data[i]->GetI0At1(defIm);
      const Real *im = defIm.getDataPointer();
      for (long j = 0; j < n; ++j) avg[j] += im[j] * weights[i];
    }
  };
  thread_mean();
  for (int iter = 0; iter < iters; ++iter) {
    for (int i = 0; i < ns; ++i) {
      data[i]->SetCurIter(iter);
      if (iter == 0) iterator.UpdateStepSizeNextIteration();
      iterator.Iterate(*data[i]);
      if (energies) energies[(long)iter * ns + i] = data[i]->GetEnergyHistory().LastEnergy()->GetEnergy();
    }
    if ((iter + 1) % mean_period == 0) thread_mean();
  }
  from_im(mean, mean_out);
  for (int i = 0; i < ns; ++i) {
    float *o = h_out + (long)i * 3 * n;
    from_vf(data[i]->Def1To0(), o, o + n, o + 2 * n);
  }
  for (auto *d : data) delete d;
  for (auto *im : ims) delete im;
  GUARD_END
}

/* ImageUtils::gaussianDownsample (MultiscaleManager::DownsampleToLevel) */
int awref_downsample(const float *in, int nx, int ny, int nz, double spx, double spy, double spz,
                     float *out, int mx, int my, int mz) {
  GUARD_BEGIN
  RealImage I(SizeType(nx, ny, nz), OriginType(0, 0, 0), SpacingType(spx, spy, spz));
  to_im(in, I);
  RealImage O;
  ImageUtils::gaussianDownsample(I, O, Vector3D<unsigned int>(mx, my, mz));
  from_im(O, out);
  GUARD_END
}

/* hToVelocity + resampleNew(CLAMP, rescale) + velocityToH, the deformation
 * upsampling of GreedyDeformationData::SetScaleLevel */
int awref_upsample_hfield(const float *h, int nx, int ny, int nz, float *out, int mx, int my,
                          int mz, int rescale) {
  GUARD_BEGIN
  VectorField f(nx, ny, nz);
  const long n = (long)nx * ny * nz, m = (long)mx * my * mz;
  to_vf(h, h + n, h + 2 * n, f);
  HField3DUtils::hToVelocity(f);
  VectorField t(mx, my, mz);
  HField3DUtils::resampleNew(f, t, Vector3D<unsigned int>(mx, my, mz),
                             HField3DUtils::BACKGROUND_STRATEGY_CLAMP, rescale != 0);
  HField3DUtils::velocityToH(t);
  from_vf(t, out, out + m, out + 2 * m);
  GUARD_END
}

/*
 * LDMM registration through LDMMIteratorCPU, scale loop of LDMMWarp::RunWarp
 * at one scale level (factor 1). use_new selects IterateNew (splatting) over
 * the default IterateOrig (Jacobian). v is [T][3][N]: read as the initial
 * velocity when v_init is set (else zero), written back at the end.
 * energies[] receives the image energy of each iteration when debug is set.
 */
int awref_ldmm_run(const float *i0, const float *i1, int nx, int ny, int nz, double spx,
                   double spy, double spz, int T, int iters, float sigma, float step,
                   int adaptive, float max_pert, double alpha, double beta, double gamma,
                   int use_new, int debug, int v_init, float *v, double *energies,
                   float *step_out, double *vec_energies) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<LDMMWarpParameterFile><LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><LDMMIterator>" << diffoper_xml(alpha, beta, gamma) << "<Sigma val=\""
      << sigma << "\"/><StepSize val=\"" << step << "\"/><UseAdaptiveStepSize val=\""
      << (adaptive ? "true" : "false") << "\"/><MaxPert val=\"" << max_pert
      << "\"/></LDMMIterator><NIterations val=\"" << iters
      << "\"/></LDMMScaleLevel><NTimeSteps val=\"" << T
      << "\"/><AutoStepReduce val=\"false\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i0, I0);
  to_im(i1, I1);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  LDMMDeformationData data(&I0, &I1, param);
  LDMMIteratorNewCPU iterator(size, origin, sp, T, debug != 0, use_new != 0);
  const long n = (long)nx * ny * nz;
  data.InitializeWarp();
  scaleManager.SetScaleLevel(0);
  const LDMMScaleLevelParam &lp = param.GetScaleLevel(0);
  iterator.SetScaleLevel(scaleManager, lp.Iterator());
  data.SetScaleLevel(scaleManager);
  data.StepSize(lp.Iterator().StepSize());
  if (v_init)
    for (int t = 0; t < T; ++t)
      to_vf(v + t * 3 * n, v + t * 3 * n + n, v + t * 3 * n + 2 * n, data.v(t));
  for (int iter = 0; iter < iters; ++iter) {
    if (iter == 0 && lp.Iterator().UseAdaptiveStepSize()) {
      iterator.UpdateStepSizeNextIteration();
      iterator.Iterate(data);
    }
    data.SetCurIter(iter);
    iterator.Iterate(data);
    if (energies) {
      // image term sum (J0_{T-1} - I1)^2 * sp^3 (LDMMEnergy::ImageEnergy is
      // that divided by sigma^2)
      LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
      energies[iter] = e ? (double)e->ImageEnergy() * sigma * sigma : 0.0;
    }
    if (vec_energies) {
      // LDMMEnergy::VecEnergy is the float sum of the step energies / T
      LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
      vec_energies[iter] = e ? (double)e->VecEnergy() * T : 0.0;
    }
  }
  for (int t = 0; t < T; ++t)
    from_vf(data.v(t), v + t * 3 * n, v + t * 3 * n + n, v + t * 3 * n + 2 * n);
  if (step_out) *step_out = data.StepSize();
  GUARD_END
}

/*
 * LDMMDeformationData::GetI1At0 and LDMMIteratorCPU::ComputeJacDet for
 * given velocities v [T][3][N] (jd may be NULL).
 */
int awref_ldmm_i1_at_0(const float *i1, const float *v, int nx, int ny, int nz, double spx,
                       double spy, double spz, int T, float *img, float *jd) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml << "<LDMMWarpParameterFile><LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><LDMMIterator>" << diffoper_xml(0.01, 0.01, 0.001)
      << "</LDMMIterator><NIterations val=\"1\"/></LDMMScaleLevel><NTimeSteps val=\"" << T
      << "\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i1, I0);
  to_im(i1, I1);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  LDMMDeformationData data(&I0, &I1, param);
  LDMMIteratorNewCPU iterator(size, origin, sp, T, false, false);
  const long n = (long)nx * ny * nz;
  data.InitializeWarp();
  scaleManager.SetScaleLevel(0);
  iterator.SetScaleLevel(scaleManager, param.GetScaleLevel(0).Iterator());
  data.SetScaleLevel(scaleManager);
  for (int t = 0; t < T; ++t)
    to_vf(v + t * 3 * n, v + t * 3 * n + n, v + t * 3 * n + 2 * n, data.v(t));
  RealImage def(size, origin, sp);
  data.GetI1At0(def);
  from_im(def, img);
  if (jd) {
    RealImage jac(size, origin, sp);
    iterator.ComputeJacDet(data.v(), &jac);
    from_im(jac, jd);
  }
  GUARD_END
}

/*
 * LDMM relaxation atlas: the AtlasThreadMain loop (Algorithms/Common/
 * AtlasThread.txx:97-181) with the LDMM thread's hooks
 * (LDMM/LDMMAtlasThreadCPU.cxx): every subject is an LDMMDeformationData
 * with I0 = the shared mean (not rescaled, as LDMMAtlasDefDataCPU) and I1 =
 * its image, one LDMMIteratorCPU per subject (one thread per image, the
 * default); BeginImageIteration's step-size pass at iteration 0; the mean
 * after every iteration from GetI1At0 and ComputeJacDet
 * (ComputeThreadMean, :207-264, JacobianScale: sum w I1At0 JacDet /
 * sum w JacDet, LDMMAtlasBuilder.txx:274-335), thread sums added in
 * subject order. mean out; v out as [ns][T][3][N]; energies[iter][i] = the
 * image term of each subject's last iteration.
 */
int awref_ldmm_atlas_run(const float *imgs, int ns, const float *weights, int nx, int ny, int nz,
                         double spx, double spy, double spz, int T, int iters, float sigma,
                         float step, int adaptive, float max_pert, double alpha, double beta,
                         double gamma, int use_new, int jacobian_scale, float *mean_out,
                         float *v_out, double *energies) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<LDMMWarpParameterFile><LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><LDMMIterator>" << diffoper_xml(alpha, beta, gamma) << "<Sigma val=\""
      << sigma << "\"/><StepSize val=\"" << step << "\"/><UseAdaptiveStepSize val=\""
      << (adaptive ? "true" : "false") << "\"/><MaxPert val=\"" << max_pert
      << "\"/></LDMMIterator><NIterations val=\"" << iters
      << "\"/></LDMMScaleLevel><NTimeSteps val=\"" << T
      << "\"/><AutoStepReduce val=\"false\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  const long n = (long)nx * ny * nz;
  RealImage mean(size, origin, sp);
  std::vector<RealImage *> I(ns);
  std::vector<LDMMDeformationData *> data(ns);
  std::vector<LDMMIteratorNewCPU *> it(ns);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  scaleManager.SetScaleLevel(0);
  const LDMMScaleLevelParam &lp = param.GetScaleLevel(0);
  for (int i = 0; i < ns; ++i) {
    I[i] = new RealImage(size, origin, sp);
    to_im(imgs + i * n, *I[i]);
    data[i] = new LDMMDeformationData(&mean, I[i], param);
    data[i]->ScaleI0(false);
    it[i] = new LDMMIteratorNewCPU(size, origin, sp, T, true, use_new != 0);
    data[i]->InitializeWarp();
    it[i]->SetScaleLevel(scaleManager, lp.Iterator());
    data[i]->SetScaleLevel(scaleManager);
    data[i]->StepSize(lp.Iterator().StepSize());
  }
  RealImage def(size, origin, sp), jac(size, origin, sp), jsum(size, origin, sp);
  auto compute_mean = [&]() {
    RealImage acc(size, origin, sp);
    acc.fill(0.0);
    jsum.fill(0.0);
    for (int i = 0; i < ns; ++i) {
      RealImage tm(size, origin, sp), tj(size, origin, sp);  // the image's thread sums
      tm.fill(0.0);
      tj.fill(0.0);
      data[i]->GetI1At0(def);
      it[i]->ComputeJacDet(data[i]->v(), &jac);
      const Real w = weights[i];
      Real *pm = tm.getDataPointer(), *pj = tj.getDataPointer();
      const Real *pd = def.getDataPointer(), *pc = jac.getDataPointer();
      for (long j = 0; j < n; ++j) {
        if (jacobian_scale) {
          pm[j] += pd[j] * pc[j] * w;
          pj[j] += pc[j] * w;
        } else {
          pm[j] += pd[j] * w;
        }
      }
      acc.pointwiseAdd(tm);
      jsum.pointwiseAdd(tj);
    }
    if (jacobian_scale) acc.pointwiseDivideBy(jsum);
    mean = acc;
  };
  compute_mean();
  for (int iter = 0; iter < iters; ++iter) {
    for (int i = 0; i < ns; ++i) {
      data[i]->SetCurIter(iter);
      if (iter == 0 && lp.Iterator().UseAdaptiveStepSize()) {
        it[i]->UpdateStepSizeNextIteration();
        it[i]->Iterate(*data[i]);
      }
      it[i]->Iterate(*data[i]);
      if (energies) {
        LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data[i]->GetEnergyHistory().LastEnergy());
        energies[iter * ns + i] = e ? (double)e->ImageEnergy() * sigma * sigma : 0.0;
      }
    }
    compute_mean();
  }
  from_im(mean, mean_out);
  for (int i = 0; i < ns; ++i)
    for (int t = 0; t < T; ++t) {
      float *vt = v_out + ((long)i * T + t) * 3 * n;
      from_vf(data[i]->v(t), vt, vt + n, vt + 2 * n);
    }
  for (int i = 0; i < ns; ++i) {
    delete it[i];
    delete data[i];
    delete I[i];
  }
  GUARD_END
}

/*
 * LDMM geodesic shooting: LDMMShootingDefData + LDMMShootingIteratorCPU at
 * one scale level, `iters` iterations from alpha0 = 0. Writes alpha0, phi0T,
 * phiT0 ([3][N] each) and the image term of each iteration's energy.
 */
int awref_shoot_run(const float *i0, const float *i1, int nx, int ny, int nz, double spx,
                    double spy, double spz, int T, int iters, float sigma, float step, double alpha,
                    double beta, double gamma, float *alpha0, float *phi0T, float *phiT0,
                    double *energies, double *vec_energies) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<LDMMWarpParameterFile><LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><LDMMIterator>" << diffoper_xml(alpha, beta, gamma) << "<Sigma val=\""
      << sigma << "\"/><StepSize val=\"" << step
      << "\"/><UseAdaptiveStepSize val=\"false\"/></LDMMIterator><NIterations val=\"" << iters
      << "\"/></LDMMScaleLevel><NTimeSteps val=\"" << T
      << "\"/><AutoStepReduce val=\"false\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i0, I0);
  to_im(i1, I1);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  LDMMShootingDefData data(&I0, &I1, param);
  LDMMShootingIteratorCPU iterator(size, origin, sp, T, true);
  const long n = (long)nx * ny * nz;
  data.InitializeWarp();
  scaleManager.SetScaleLevel(0);
  const LDMMScaleLevelParam &lp = param.GetScaleLevel(0);
  iterator.SetScaleLevel(scaleManager, lp.Iterator());
  // the const overload: LDMMShootingDefData.h declares a non-const one that
  // has no definition
  data.SetScaleLevel(static_cast<const MultiscaleManager &>(scaleManager));
  data.StepSize(lp.Iterator().StepSize());
  for (int iter = 0; iter < iters; ++iter) {
    data.SetCurIter(iter);
    iterator.Iterate(data);
    if (energies) {
      LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
      energies[iter] = e ? (double)e->ImageEnergy() * sigma * sigma : 0.0;
    }
    if (vec_energies) {
      LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
      double sum = 0.0;
      for (int t = 0; e && t < T; ++t) sum += (double)e->VecStepEnergy(t);
      vec_energies[iter] = sum;
    }
  }
  from_im(data.Alpha0(), alpha0);
  from_vf(data.Phi0T(), phi0T, phi0T + n, phi0T + 2 * n);
  from_vf(data.PhiT0(), phiT0, phiT0 + n, phiT0 + 2 * n);
  GUARD_END
}

// LDMMWarpAd<LDMMAdShootingIteratorCPU>::RunWarp (LDMM/LDMMWarp.txx:72-133
// with LDMMWarpAd.txx:37-42): every scale level in the given order (the
// parameter file's; the MultiscaleManager sorts them), fixed step per level,
// then FinishWarp's final maps. energies: per iteration the raw image term
// and <L v0, v0>.
int awref_adshoot_run(const float *i0, const float *i1, int nx, int ny, int nz, double spx,
                      double spy, double spz, int T, int nscales, const int *factors,
                      const int *iters, const float *steps, float sigma, double alpha,
                      double beta, double gamma, float *alpha0, float *phi0T, float *phiT0,
                      double *img_energy, double *vec_energy) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<LDMMWarpParameterFile>";
  for (int s = 0; s < nscales; ++s)
    xml << "<LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"" << factors[s]
        << "\"/></ScaleLevel><LDMMIterator>" << diffoper_xml(alpha, beta, gamma)
        << "<Sigma val=\"" << sigma << "\"/><StepSize val=\"" << steps[s]
        << "\"/><UseAdaptiveStepSize val=\"false\"/></LDMMIterator><NIterations val=\""
        << iters[s] << "\"/></LDMMScaleLevel>";
  xml << "<NTimeSteps val=\"" << T << "\"/><AutoStepReduce val=\"false\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i0, I0);
  to_im(i1, I1);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  LDMMShootingDefData data(&I0, &I1, param);
  LDMMAdShootingIteratorCPU iterator(size, origin, sp, T, true);
  const long n = (long)nx * ny * nz;
  data.InitializeWarp();
  int e = 0;
  for (unsigned level = 0; level < param.GetNumberOfScaleLevels(); ++level) {
    scaleManager.SetScaleLevel(level);
    const LDMMScaleLevelParam &lp = param.GetScaleLevel(level);
    iterator.SetScaleLevel(scaleManager, lp.Iterator());
    data.SetScaleLevel(static_cast<const MultiscaleManager &>(scaleManager));
    data.StepSize(lp.Iterator().StepSize());
    for (unsigned iter = 0; iter < lp.NIterations(); ++iter, ++e) {
      data.SetCurIter(iter);
      iterator.Iterate(data);
      LDMMEnergy *en = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
      if (img_energy) img_energy[e] = en ? (double)en->ImageEnergy() * sigma * sigma : 0.0;
      if (vec_energy) vec_energy[e] = en ? (double)en->VecStepEnergy(0) : 0.0;
    }
  }
  iterator.finalUpdatePhi0T(data);
  iterator.finalUpdatePhiT0(data);
  from_im(data.Alpha0(), alpha0);
  from_vf(data.Phi0T(), phi0T, phi0T + n, phi0T + 2 * n);
  from_vf(data.PhiT0(), phiT0, phiT0 + n, phiT0 + 2 * n);
  GUARD_END
}

// MedianCalculator::Select over n images stacked [n][nvox]: the per-voxel
// k-th smallest value (the UsePerVoxelMedian atlas); 1 when it throws
int awref_voxel_median(const float *imgs, int n, int nx, int ny, int nz, int k, float *out) {
  GUARD_BEGIN
  SizeType size(nx, ny, nz);
  OriginType origin(0, 0, 0);
  SpacingType sp(1, 1, 1);
  const long nvox = (long)nx * ny * nz;
  std::vector<RealImage *> ims;
  for (int m = 0; m < n; ++m) {
    ims.push_back(new RealImage(size, origin, sp));
    to_im(imgs + m * nvox, *ims.back());
  }
  RealImage rtn(size, origin, sp);
  int rc = 0;
  try {
    MedianCalculator::Select(ims, (unsigned)k, rtn);
  } catch (...) {
    rc = 1;
  }
  for (RealImage *im : ims) delete im;
  if (rc) return 1;
  from_im(rtn, out);
  GUARD_END
}

// LDMMGeodesicShootingCPU::ShootImage(I0, alpha0, T): the final image and
// both maps
int awref_geodesic_shoot(const float *i0, const float *a0, int nx, int ny, int nz, double spx,
                         double spy, double spz, int T, double alpha, double beta, double gamma,
                         float *phi0T, float *phiT0, float *img) {
  GUARD_BEGIN
  DiffOperParam param;
  parse_into(param, diffoper_xml(alpha, beta, gamma));
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), A0(size, origin, sp);
  to_im(i0, I0);
  to_im(a0, A0);
  LDMMGeodesicShootingCPU shooter(size, sp, param);
  shooter.ShootImage(I0, A0, (unsigned)T);
  const long n = (long)nx * ny * nz;
  from_vf(shooter.GetPhi0To1(), phi0T, phi0T + n, phi0T + 2 * n);
  from_vf(shooter.GetPhi1To0(), phiT0, phiT0 + n, phiT0 + 2 * n);
  from_im(shooter.GetFinalImage(), img);
  GUARD_END
}

// LDMMVelShootingIteratorCPU driven through the LDMMWarp loop at one scale:
// v0 (3N) after iters iterations (the step-size pass first when adaptive),
// both maps of the last, per iteration the raw image term and the sum of
// the step energies; step_out the step used
int awref_velshoot_run(const float *i0, const float *i1, int nx, int ny, int nz, double spx,
                       double spy, double spz, int T, int iters, float sigma, float step,
                       int adaptive, float max_pert, double alpha, double beta, double gamma,
                       float *v0, float *phi0T, float *phiT0, double *energies,
                       double *vec_energies, float *step_out) {
  GUARD_BEGIN
  std::ostringstream xml;
  xml.precision(17);
  xml << "<LDMMWarpParameterFile><LDMMScaleLevel><ScaleLevel><DownsampleFactor val=\"1\"/>"
      << "</ScaleLevel><LDMMIterator>" << diffoper_xml(alpha, beta, gamma) << "<Sigma val=\""
      << sigma << "\"/><StepSize val=\"" << step << "\"/><UseAdaptiveStepSize val=\""
      << (adaptive ? "true" : "false") << "\"/><MaxPert val=\"" << max_pert
      << "\"/></LDMMIterator><NIterations val=\"" << iters
      << "\"/></LDMMScaleLevel><NTimeSteps val=\"" << T
      << "\"/><AutoStepReduce val=\"false\"/></LDMMWarpParameterFile>";
  LDMMParam param;
  parse_into(param, xml.str());
  SizeType size(nx, ny, nz);
  SpacingType sp(spx, spy, spz);
  OriginType origin(0, 0, 0);
  RealImage I0(size, origin, sp), I1(size, origin, sp);
  to_im(i0, I0);
  to_im(i1, I1);
  MultiscaleManager scaleManager(size, sp, origin, param);
  scaleManager.SetScaleVectorFields(false);
  LDMMVelShootingDefData data(&I0, &I1, param);
  LDMMVelShootingIteratorCPU iterator(size, origin, sp, T, true);
  const long n = (long)nx * ny * nz;
  data.InitializeWarp();
  scaleManager.SetScaleLevel(0);
  const LDMMScaleLevelParam &lp = param.GetScaleLevel(0);
  iterator.SetScaleLevel(scaleManager, lp.Iterator());
  data.SetScaleLevel(static_cast<const MultiscaleManager &>(scaleManager));
  data.StepSize(lp.Iterator().StepSize());
  for (int iter = 0; iter < iters; ++iter) {
    if (iter == 0 && lp.Iterator().UseAdaptiveStepSize()) {
      iterator.UpdateStepSizeNextIteration();
      iterator.Iterate(data);
    }
    data.SetCurIter(iter);
    iterator.Iterate(data);
    LDMMEnergy *e = dynamic_cast<LDMMEnergy *>(data.GetEnergyHistory().LastEnergy());
    if (energies) energies[iter] = e ? (double)e->ImageEnergy() * sigma * sigma : 0.0;
    if (vec_energies) {
      double sum = 0.0;
      for (int t = 0; e && t < T; ++t) sum += (double)e->VecStepEnergy(t);
      vec_energies[iter] = sum;
    }
  }
  from_vf(data.V0(), v0, v0 + n, v0 + 2 * n);
  from_vf(data.Phi0T(), phi0T, phi0T + n, phi0T + 2 * n);
  from_vf(data.PhiT0(), phiT0, phiT0 + n, phiT0 + 2 * n);
  if (step_out) *step_out = data.StepSize();
  GUARD_END
}

}  // extern "C"
