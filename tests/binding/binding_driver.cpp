// binding_driver.cpp — runs the reference-side bindings (include/aw_b200_*.hpp)
// over the stand-in headers of this directory, the way GreedyWarp::RunWarp
// (Greedy/GreedyWarp.txx:71-125) and LDMMWarp::RunWarp (LDMM/LDMMWarp.txx:
// 71-130) drive their iterators at one scale level. Test infrastructure:
// reads raw float32 inputs from a directory, writes raw outputs there.
//
//   binding_driver greedy   <dir> nx ny nz iters inverse
//   binding_driver ldmm     <dir> nx ny nz T iters
//   binding_driver diffoper <dir> nx ny nz inverse
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "aw_b200_diffoper.hpp"
#include "aw_b200_greedy_iterator.hpp"
#include "aw_b200_ldmm_iterator.hpp"

namespace {

std::vector<float> read_raw(const std::string &path, size_t n) {
  std::vector<float> a(n);
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f || std::fread(a.data(), sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", path.c_str());
    std::exit(2);
  }
  std::fclose(f);
  return a;
}

void write_raw(const std::string &path, const float *a, size_t n) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(a, sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fclose(f);
}

float *to_device(const std::vector<float> &a) {
  float *d = nullptr;
  if (cudaMalloc((void **)&d, a.size() * sizeof(float)) != cudaSuccess ||
      cudaMemcpy(d, a.data(), a.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    std::fprintf(stderr, "device allocation failed\n");
    std::exit(3);
  }
  return d;
}

std::vector<float> to_host(const float *d, size_t n) {
  std::vector<float> a(n);
  if (cudaMemcpy(a.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "device read failed\n");
    std::exit(3);
  }
  return a;
}

// identity deformation, three planes, x fastest
std::vector<float> identity(unsigned nx, unsigned ny, unsigned nz) {
  const size_t n = (size_t)nx * ny * nz;
  std::vector<float> h(3 * n);
  for (unsigned z = 0; z < nz; ++z)
    for (unsigned y = 0; y < ny; ++y)
      for (unsigned x = 0; x < nx; ++x) {
        const size_t i = ((size_t)z * ny + y) * nx + x;
        h[i] = (float)x;
        h[n + i] = (float)y;
        h[2 * n + i] = (float)z;
      }
  return h;
}

cplVector3DArray planes(float *base, size_t n) {
  cplVector3DArray a;
  a.x = base;
  a.y = base + n;
  a.z = base + 2 * n;
  return a;
}

void write_energies(const std::string &path, const std::vector<Real> &e) {
  write_raw(path, e.data(), e.size());
}

int run_greedy(const std::string &dir, SizeType size, int iters, bool inverse) {
  const size_t n = (size_t)size.x * size.y * size.z;
  SpacingType sp{1.0, 1.0, 1.0};
  OriginType origin{0, 0, 0};
  float *I0 = to_device(read_raw(dir + "/I0.raw", n));
  float *I1 = to_device(read_raw(dir + "/I1.raw", n));
  float *h = to_device(identity(size.x, size.y, size.z));
  float *hi = to_device(identity(size.x, size.y, size.z));
  GreedyDeformationDataGPU data(size, sp, I0, I1, planes(h, n), planes(hi, n), inverse);
  MultiscaleManager scale(size, sp);
  GreedyIteratorParam param(KernelParam(DiffOperParam()), 0.5f);
  GreedyIteratorB200 it(size, origin, sp, true);
  it.SetScaleLevel(scale, param);
  for (int k = 0; k < iters; ++k) {
    if (k == 0) it.UpdateStepSizeNextIteration();
    it.Iterate(data);
  }
  write_raw(dir + "/h.raw", to_host(h, 3 * n).data(), 3 * n);
  if (inverse) write_raw(dir + "/hinv.raw", to_host(hi, 3 * n).data(), 3 * n);
  write_energies(dir + "/energies.raw", data.mEnergies);
  const float step = data.StepSize();
  write_raw(dir + "/step.raw", &step, 1);
  return 0;
}

int run_ldmm(const std::string &dir, SizeType size, unsigned T, int iters) {
  const size_t n = (size_t)size.x * size.y * size.z;
  SpacingType sp{1.0, 1.0, 1.0};
  OriginType origin{0, 0, 0};
  float *I0 = to_device(read_raw(dir + "/I0.raw", n));
  float *I1 = to_device(read_raw(dir + "/I1.raw", n));
  // the data object's T fields, each in an allocation of its own
  std::vector<cplVector3DArray> v(T);
  std::vector<float *> vbase(T);
  for (unsigned t = 0; t < T; ++t) {
    vbase[t] = to_device(std::vector<float>(3 * n, 0.0f));
    v[t] = planes(vbase[t], n);
  }
  LDMMDeformationDataGPU data(size, sp, I0, I1, v);
  MultiscaleManager scale(size, sp);
  LDMMIteratorParam param(KernelParam(DiffOperParam()), 1.0f, 0.01f, 0.1f);
  LDMMIteratorB200 it(size, origin, sp, T, true);
  it.SetScaleLevel(scale, param);
  data.StepSize(param.StepSize());
  for (int k = 0; k < iters; ++k) it.Iterate(data);
  std::vector<float> vout(3 * n * T);
  for (unsigned t = 0; t < T; ++t) {
    std::vector<float> a = to_host(vbase[t], 3 * n);
    std::copy(a.begin(), a.end(), vout.begin() + 3 * n * t);
  }
  write_raw(dir + "/v.raw", vout.data(), vout.size());
  it.Iterate(data, true);
  std::vector<float> al(n * T);
  for (unsigned t = 0; t < T; ++t) {
    std::vector<float> a = to_host(it.GetAlpha(t), n);
    std::copy(a.begin(), a.end(), al.begin() + n * t);
  }
  write_raw(dir + "/alphas.raw", al.data(), al.size());
  float *jac = to_device(std::vector<float>(n, 0.0f));
  it.ComputeJacDet(data.dV(), jac);
  write_raw(dir + "/jacdet.raw", to_host(jac, n).data(), n);
  write_energies(dir + "/energies.raw", data.mEnergies);
  return 0;
}

int run_diffoper(const std::string &dir, SizeType size, bool inverse) {
  const size_t n = (size_t)size.x * size.y * size.z;
  float *f = to_device(read_raw(dir + "/f.raw", 3 * n));
  cplVector3DArray a = planes(f, n);
  DiffOperB200 op;
  op.SetSize(size, SpacingType{1.0, 1.3, 0.8}, KernelParam(DiffOperParam()));
  if (inverse)
    op.ApplyInverseOperator(a);
  else
    op.ApplyOperator(a);
  write_raw(dir + "/out.raw", to_host(f, 3 * n).data(), 3 * n);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s greedy|ldmm|diffoper dir nx ny nz ...\n", argv[0]);
    return 1;
  }
  const std::string mode = argv[1], dir = argv[2];
  SizeType size{(unsigned)std::atoi(argv[3]), (unsigned)std::atoi(argv[4]),
                (unsigned)std::atoi(argv[5])};
  try {
    if (mode == "greedy" && argc == 8) return run_greedy(dir, size, std::atoi(argv[6]),
                                                         std::atoi(argv[7]) != 0);
    if (mode == "ldmm" && argc == 8) return run_ldmm(dir, size, (unsigned)std::atoi(argv[6]),
                                                     std::atoi(argv[7]));
    if (mode == "diffoper" && argc == 7) return run_diffoper(dir, size, std::atoi(argv[6]) != 0);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 4;
  }
  std::fprintf(stderr, "bad arguments\n");
  return 1;
}
