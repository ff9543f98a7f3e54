// The 2D swimmer-ISF table (layout and interpolation: isf.cuh), built on the
// device once per device, and ddm_isf_eval, the C-ABI view of both swimmer
// kernels as the fits evaluate them.
//
// Node values: P_Z(cos th) and dP/dth from Laplace's first integral,
//   P_Z(cos th) = (1/pi) int_0^pi Re (cos th + i sin th cos phi)^Z dphi,
// by the trapezoid rule (the integrand is smooth, even and 2 pi periodic in
// phi, so the rule converges exponentially); dP/dth differentiates under the
// integral. The node count grows with the phase Z th and with 1/cos th (the
// integrand passes close to its branch point when cos th is small):
// 24 + 2 ceil(Z th) + ceil(4 / cos th) nodes, at most 65536 -- about 1e-11
// against an adaptive quadrature of the Schulz average of J0. One warp per
// table node, lanes split the quadrature, FP64 throughout.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "isf.cuh"

namespace ddm {

namespace {

static __device__ __align__(256) double2 g_isf2d_node[ISF2D_MAX_NODES];
static __device__ __align__(256) double4 g_isf2d_row[ISF2D_ROWS];

__global__ void __launch_bounds__(256) isf2d_build_kernel(int nrows) {
  const int row = blockIdx.x;
  if (row >= nrows) return;
  const double4 r = g_isf2d_row[row];
  const double Z = r.x, h = r.y, th_end = r.z;
  const int m = (int)(th_end / h + 0.5), base = (int)r.w;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = warp; j <= m; j += blockDim.x >> 5) {
    const double th = j == m ? th_end : j * h;
    double s, c;
    sincos(th, &s, &c);
    const double nn = 24.0 + 2.0 * ceil(Z * th) + ceil(4.0 / fmax(c, 1e-12));
    const int n = nn > 65536.0 ? 65536 : (int)nn;
    double sv = 0.0, sd = 0.0;
    for (int k = lane; k <= n; k += 32) {
      const double cp = cospi((double)k / n);
      const double wr = c, wi = s * cp;         // w = cos th + i sin th cos phi
      const double dr = -s, di = c * cp;        // dw/dth
      const double m2 = wr * wr + wi * wi;
      const double arg = atan2(wi, wr);
      const double mag = exp(0.5 * Z * log(m2));
      double sn, cs;
      sincos(Z * arg, &sn, &cs);
      const double pr = mag * cs, pi = mag * sn;  // w^Z
      // Z w^Z (dw/dth) / w = Z w^Z (dw/dth) conj(w) / |w|^2
      const double qr = (dr * wr + di * wi) / m2, qi = (di * wr - dr * wi) / m2;
      const double wt = (k == 0 || k == n) ? 0.5 : 1.0;
      sv += wt * pr;
      sd += wt * Z * (pr * qr - pi * qi);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sv += __shfl_xor_sync(0xffffffffu, sv, o);
      sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if (lane == 0) g_isf2d_node[base + j] = make_double2(sv / n, sd / n);
  }
}

struct TableState {
  bool ready = false;
  Isf2dTable t{};
};
std::mutex g_mu;
std::vector<TableState> g_tables;

}  // namespace

cudaError_t isf2d_table(Isf2dTable* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_tables.size() <= dev) g_tables.resize(dev + 1);
  TableState& st = g_tables[dev];
  if (!st.ready) {
    // rows: Z_i = exp(ln 0.5 + i dlz); th from 0 to th_end = acos(e^(-25/(Z+1)))
    // in m steps of at most min(0.02, 0.08 / (Z + 1/2))
    const double lz0 = std::log(ISF2D_ZMIN), dlz = (std::log(ISF2D_ZMAX) - lz0) / (ISF2D_ROWS - 1);
    std::vector<double4> rows(ISF2D_ROWS);
    int total = 0;
    for (int i = 0; i < ISF2D_ROWS; i++) {
      const double Z = std::exp(lz0 + i * dlz);
      const double th_end = std::acos(std::exp(-25.0 / (Z + 1.0)));
      const double h0 = std::fmin(0.02, 0.08 / (Z + 0.5));
      const int m = (int)std::ceil(th_end / h0);
      rows[i] = make_double4(Z, th_end / m, th_end, (double)total);
      total += m + 1;
    }
    if (total > ISF2D_MAX_NODES) return cudaErrorInvalidValue;
    double2* node = nullptr;
    double4* row = nullptr;
    if ((e = cudaGetSymbolAddress((void**)&node, g_isf2d_node)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress((void**)&row, g_isf2d_row)) != cudaSuccess) return e;
    cudaStream_t s = nullptr;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return e;
    e = cudaMemcpyAsync(row, rows.data(), sizeof(double4) * ISF2D_ROWS, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      isf2d_build_kernel<<<ISF2D_ROWS, 256, 0, s>>>(ISF2D_ROWS);
      e = cudaGetLastError();
    }
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return e;
    st.t.node = node;
    st.t.row = row;
    st.t.lz0 = lz0;
    st.t.dlz = dlz;
    st.ready = true;
  }
  *out = st.t;
  return cudaSuccess;
}

namespace {

__global__ void isf_eval_kernel(int n, int geometry2d, Isf2dTable t, const double* __restrict__ x,
                                const double* __restrict__ Z, double* __restrict__ g, double* __restrict__ gx,
                                double* __restrict__ gz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a, b, c;
  if (geometry2d)
    isf2d_d(t, x[i], Z[i], a, b, c);
  else
    isf3d_d<double>(x[i], Z[i], a, b, c);
  g[i] = a;
  if (gx) gx[i] = b;
  if (gz) gz[i] = c;
}

}  // namespace

}  // namespace ddm

extern std::string& ddm_detached_error();  // message slot of calls without an engine (engine.cu)

extern "C" int ddm_isf_eval(int32_t n, int32_t geometry2d, const double* x, const double* Z, double* g,
                            double* xdgdx, double* Zdgdz) {
  ddm_detached_error().clear();
  if (n < 0 || !(geometry2d == 0 || geometry2d == 1)) {
    ddm_detached_error() = "ddm_isf_eval: need n >= 0 and geometry2d 0 or 1";
    return DDM_ERR_ARG;
  }
  if (n == 0) return DDM_OK;
  if (!x || !Z || !g) {
    ddm_detached_error() = "ddm_isf_eval: null array";
    return DDM_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    ddm_detached_error() = "ddm_isf_eval: no CUDA device";
    return DDM_ERR_NODEV;
  }
  ddm::Isf2dTable t{};
  cudaError_t e = ddm::isf2d_table(&t);
  double* buf = nullptr;
  const size_t nb = sizeof(double) * n;
  if (e == cudaSuccess) e = cudaMalloc((void**)&buf, 5 * nb);
  if (e == cudaSuccess) e = cudaMemcpy(buf, x, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(buf + n, Z, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    ddm::isf_eval_kernel<<<(n + 255) / 256, 256>>>(n, geometry2d, t, buf, buf + n, buf + 2 * (size_t)n,
                                                    buf + 3 * (size_t)n, buf + 4 * (size_t)n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(g, buf + 2 * (size_t)n, nb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && xdgdx) e = cudaMemcpy(xdgdx, buf + 3 * (size_t)n, nb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && Zdgdz) e = cudaMemcpy(Zdgdz, buf + 4 * (size_t)n, nb, cudaMemcpyDeviceToHost);
  if (buf) cudaFree(buf);
  if (e != cudaSuccess) {
    ddm_detached_error() = std::string("ddm_isf_eval: ") + cudaGetErrorString(e);
    return DDM_ERR_CUDA;
  }
  return DDM_OK;
}
