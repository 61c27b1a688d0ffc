// Legacy VTK output of the surface (FastScape_VTK).
//
// Reference: Make_VTK, src/FastScape_ctx.f90:692-777 (FastScape_VTK,
// src/FastScape_api.f90:728-741).  One file per call, <dir>/Topography<step>.vtk
// with the step zero-padded to 7 digits; with vex < 0 also Basement<step>.vtk
// and SeaLevel<step>.vtk.  Each file is the legacy "BINARY" STRUCTURED_GRID
// format: an ASCII header, float32 points (dx*(i-1), dy*(j-1), z*|vex|) with x
// fastest, "POINT_DATA", then SCALARS blocks named H (or B) and HHHHH (the
// caller's field f), or SL.  The reference writes it as one direct-access
// unformatted record built with -fconvert=big-endian (CMakeLists.txt:49), so
// every float is big-endian IEEE single (the double rounded to nearest).
//
// The device packs the floats (rounding, byte order, point coordinates) into
// free scratch in one kernel; one copy brings them to the host, which writes
// the header strings around them.
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fastscape_b200.h"
#include "fsb_kernels.cuh"

namespace fsb {

namespace {

__device__ inline unsigned be32(double v) { return __byte_perm(__float_as_uint(__double2float_rn(v)), 0, 0x0123); }

// out[0..3nn): points; out[3nn..4nn): s1; out[4nn..5nn): s2 (when given).
// z == nullptr means z = zc everywhere (the sea-level surface); s1 == nullptr
// means s1 = s1c everywhere.
__global__ void k_vtk_pack(int nx, int ny, double dx, double dy, double avex, const double* __restrict__ z, double zc,
                           const double* __restrict__ s1, double s1c, const double* __restrict__ s2,
                           unsigned* __restrict__ out) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    out[3 * (size_t)k] = be32(dx * (double)i);
    out[3 * (size_t)k + 1] = be32(dy * (double)j);
    out[3 * (size_t)k + 2] = be32((z ? z[k] : zc) * avex);
    out[3 * (size_t)nn + k] = be32(s1 ? s1[k] : s1c);
    if (s2) out[4 * (size_t)nn + k] = be32(s2[k]);
  }
}

std::string fmt_int(const char* f, long long v) {
  char b[32];
  std::snprintf(b, sizeof b, f, v);
  return b;
}

}  // namespace

// Writes one file; `name` is the scalar block name of s1 ("H", "B", "SL");
// s2 (the caller's field, block "HHHHH") may be null (sea-level file).
static int vtk_file(Ctx& c, const std::string& path, const double* z, double zc, const char* name,
                    const double* s1, double s1c, const double* s2, double vex) {
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  unsigned* dev = static_cast<unsigned*>(c.mfd_line);  // 128 bytes per node, free between steps
  k_vtk_pack<<<grid1d(nn), kBlock, 0, c.stream>>>(nx, ny, dx, dy, std::fabs(vex), z, zc, s1, s1c, s2, dev);
  c.count_launch();
  const size_t nflt = (s2 ? 5 : 4) * (size_t)nn;
  std::vector<unsigned> host(nflt);
  if (cudaMemcpyAsync(host.data(), dev, sizeof(unsigned) * nflt, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess)
    return report_error("VTK: copying the packed fields failed");
  const std::string nnc = fmt_int("%12lld", nn);
  const std::string header = std::string("# vtk DataFile Version 3.0\nFastScape\nBINARY\nDATASET STRUCTURED_GRID\n") +
                             "DIMENSIONS " + fmt_int("%6lld", nx) + " " + fmt_int("%6lld", ny) + " 1\nPOINTS" +
                             nnc + " float\n";
  const std::string footer = "POINT_DATA" + nnc + "\n";
  const std::string part2 = " float 1\nLOOKUP_TABLE default\n";
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return report_error("VTK: cannot open " + path + ": " + std::strerror(errno));
  bool ok = std::fwrite(header.data(), 1, header.size(), fp) == header.size();
  ok = ok && std::fwrite(host.data(), 4, 3 * (size_t)nn, fp) == 3 * (size_t)nn;
  ok = ok && std::fwrite(footer.data(), 1, footer.size(), fp) == footer.size();
  const std::string b1 = std::string("SCALARS ") + name + part2;
  ok = ok && std::fwrite(b1.data(), 1, b1.size(), fp) == b1.size();
  ok = ok && std::fwrite(host.data() + 3 * (size_t)nn, 4, nn, fp) == (size_t)nn;
  if (s2) {
    const std::string b2 = std::string("SCALARS HHHHH") + part2;
    ok = ok && std::fwrite(b2.data(), 1, b2.size(), fp) == b2.size();
    ok = ok && std::fwrite(host.data() + 4 * (size_t)nn, 4, nn, fp) == (size_t)nn;
  }
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) return report_error("VTK: writing " + path + " failed");
  return 0;
}

int write_vtk(Ctx& c, const double* f_dev, double vex, const char* dir) {
  const std::string d = (dir && *dir) ? dir : "VTK";
  if (mkdir(d.c_str(), 0777) != 0 && errno != EEXIST)
    return report_error("VTK: cannot create directory " + d + ": " + std::strerror(errno));
  const std::string cstep = fmt_int("%07lld", c.step);
  if (vtk_file(c, d + "/Topography" + cstep + ".vtk", c.h, 0.0, "H", c.h, 0.0, f_dev, vex)) return 1;
  if (vex < 0.0) {
    if (vtk_file(c, d + "/Basement" + cstep + ".vtk", c.b, 0.0, "B", c.b, 0.0, f_dev, vex)) return 1;
    const double sealevel = 0.0;  // no marine component: the reference's default sea level
    if (vtk_file(c, d + "/SeaLevel" + cstep + ".vtk", nullptr, sealevel, "SL", nullptr, sealevel, nullptr, vex))
      return 1;
  }
  return 0;
}

}  // namespace fsb
