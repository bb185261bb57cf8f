/*
 * noalloc.cu — metric recovery for one small mesh without any device
 * allocation: trn_metric_noalloc (declared in include/trinity_b200.h).
 *
 * Who needs it: a caller that owns every byte of device memory itself — a
 * solver running on a fixed, pre-reserved memory budget, or one whose device
 * memory all comes from its own pool allocator — may not let a library call
 * cudaMalloc/cudaFree in the middle of its time stepping (those calls also
 * synchronise the device). Such a caller hands over its own device buffers for
 * the input and the output; everything else this computation needs lives in
 * one file-scope __device__ array below.
 *
 * The scratch array is sized for at most TRN_NOALLOC_MAX_NODES vertices,
 * TRN_NOALLOC_MAX_ELEMS triangles and TRN_NOALLOC_BUCKET triangles around one
 * vertex; it takes about 6 MB on every GPU that loads this library, for as
 * long as the process lives. Every call on a device shares it: calls that
 * overlap on the GPU (other streams, other host threads) race and corrupt
 * each other's results, so serialise them. The array keeps the last call's
 * contents; each call first clears what must start empty.
 *
 * Host code cannot use the array's name as a device address (in host code it
 * names a host-side stand-in), so the first call on each device looks the
 * address up with cudaGetSymbolAddress while that device is current and keeps
 * it.
 *
 * The computation is the same kernels, in the same order, as trn_metric_run
 * (gradient, Hessian with local L^p scaling, complexity with the fixed-shape
 * tree sum, global scaling), so the tensors are identical to it when that
 * mesh also sums with the tree (its default; exact_sum and replay sum in
 * element order). The kernels run on the caller's stream with the address
 * looked up for the current device, so the stream must belong to it.
 */
#include "trn_internal.h"
#include "trn_libm.h"
#include "../../include/trinity_b200.h"

#include <cmath>
#include <cstdio>
#include <mutex>

namespace trn {

/* kernels of topology.cu and metric.cu, reused as they are */
__global__ void k_fill_stencils(DMesh m, int nb_elems);
__global__ void k_sort_stencils(DMesh m, int nb_nodes);
__global__ void k_build_vicin(DMesh m, int nb_nodes, int only_flagged);
__global__ void k_gradient(DMesh m, int nb_nodes, const double* __restrict__ solut,
                           double2* __restrict__ grad, double* __restrict__ atot);
__global__ void k_hessian_local(DMesh m, int nb_nodes, const double2* __restrict__ grad,
                                double scale_exp, double4* __restrict__ hsym,
                                double4* __restrict__ mloc);
__global__ void k_complexity_term(DMesh m, int nb_elems, double* __restrict__ terms);
__global__ void k_sum_partial(const double* __restrict__ terms, int n, double* partial);
__global__ void k_sum_final(const double* __restrict__ partial, int nb, double* out);
__global__ void k_normalize(DMesh m, int nb_nodes, const double* complexity, double target,
                            double eig_min, double eig_max);

namespace {

constexpr size_t kMaxN = TRN_NOALLOC_MAX_NODES;
constexpr size_t kMaxE = TRN_NOALLOC_MAX_ELEMS;
constexpr size_t kB = TRN_NOALLOC_BUCKET;
constexpr size_t kPartials = 4096;  /* >= any grid_for() block count */

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t) 255; }

/* carve-up of the scratch array (byte offsets, each 256-byte aligned) */
constexpr size_t oTri = 0;
constexpr size_t oPts = oTri + align256(sizeof(int4) * kMaxE);
constexpr size_t oTen = oPts + align256(sizeof(double2) * kMaxN);
constexpr size_t oStenc = oTen + align256(sizeof(double4) * kMaxN);
constexpr size_t oVic = oStenc + align256(sizeof(int) * kMaxN * kB);
constexpr size_t oDeg = oVic + align256(sizeof(int) * kMaxN * kB);
constexpr size_t oVdeg = oDeg + align256(sizeof(int) * kMaxN);
constexpr size_t oAlive = oVdeg + align256(sizeof(int) * kMaxN);
constexpr size_t oGrad = oAlive + align256(kMaxN);
constexpr size_t oTerms = oGrad + align256(sizeof(double2) * kMaxN);
constexpr size_t oCplx = oTerms + align256(sizeof(double) * (kMaxE + kPartials));
constexpr size_t oErr = oCplx + 256;
constexpr size_t kScratchBytes = oErr + 256;

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {nullptr};

/* device address of the scratch array on the current device; looked up once */
int scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TRN_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "trn_metric_noalloc: cudaGetSymbolAddress failed: %s\n",
                   cudaGetErrorString(e));
      return TRN_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return TRN_OK;
}

__global__ void k_na_expand(const int* __restrict__ tris, int nb_elems, int nb_nodes,
                            int4* __restrict__ tri4, int* err) {
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int a = tris[3 * i], b = tris[3 * i + 1], c = tris[3 * i + 2];
    if (a < 0 || a >= nb_nodes || b < 0 || b >= nb_nodes || c < 0 || c >= nb_nodes) {
      trn_set_error(err, TRN_DERR_INVALID);
      a = b = c = -1;
    }
    tri4[i] = make_int4(a, b, c, 0);
  }
}

__global__ void k_na_points(const double* __restrict__ pts, int nb_nodes, double2* __restrict__ out) {
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride())
    out[v] = make_double2(pts[2 * v], pts[2 * v + 1]);
}

__global__ void k_na_tensor(const double4* __restrict__ ten, int nb_nodes, double* __restrict__ out) {
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    double4 t = ten[v];
    out[3 * v] = t.x;
    out[3 * v + 1] = t.y;
    out[3 * v + 2] = t.z;
  }
}

}  // namespace
}  // namespace trn

extern "C" int trn_metric_noalloc(int nb_nodes, int nb_elems, const double* d_points,
                                  const int* d_tris, const double* d_solut, double target_factor,
                                  int lp_norm, double h_min, double h_max, double* d_tensor,
                                  void* stream) {
  using namespace trn;
  if (nb_nodes <= 0 || nb_elems <= 0 || !d_points || !d_tris || !d_solut || !d_tensor ||
      lp_norm < 0 || h_min <= 0 || h_max <= 0)
    return TRN_ERR_INVALID;
  if ((size_t) nb_nodes > kMaxN || (size_t) nb_elems > kMaxE) {
    std::fprintf(stderr,
                 "trn_metric_noalloc: %d vertices / %d triangles exceed the fixed scratch "
                 "(at most %d vertices and %d triangles)\n",
                 nb_nodes, nb_elems, TRN_NOALLOC_MAX_NODES, TRN_NOALLOC_MAX_ELEMS);
    return TRN_ERR_CAPACITY;
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  DMesh d{};
  d.tri = reinterpret_cast<int4*>(base + oTri);
  d.pts = reinterpret_cast<double2*>(base + oPts);
  d.ten = reinterpret_cast<double4*>(base + oTen);
  d.stenc = reinterpret_cast<int*>(base + oStenc);
  d.vic = reinterpret_cast<int*>(base + oVic);
  d.deg = reinterpret_cast<int*>(base + oDeg);
  d.vdeg = reinterpret_cast<int*>(base + oVdeg);
  d.alive = base + oAlive;
  d.err = reinterpret_cast<int*>(base + oErr);
  d.bucket = (int) kB;
  d.capa_node = nb_nodes;
  d.capa_elem = nb_elems;
  double2* grad = reinterpret_cast<double2*>(base + oGrad);
  double* terms = reinterpret_cast<double*>(base + oTerms);
  double* cplx = reinterpret_cast<double*>(base + oCplx);

  /* what must start empty: degrees, stencil/adjacency rows, error word */
  if (cudaMemsetAsync(d.err, 0, sizeof(int), s) != cudaSuccess ||
      cudaMemsetAsync(d.deg, 0, sizeof(int) * (size_t) nb_nodes, s) != cudaSuccess ||
      cudaMemsetAsync(d.vdeg, 0, sizeof(int) * (size_t) nb_nodes, s) != cudaSuccess ||
      cudaMemsetAsync(d.stenc, 0xff, sizeof(int) * (size_t) nb_nodes * kB, s) != cudaSuccess ||
      cudaMemsetAsync(d.vic, 0xff, sizeof(int) * (size_t) nb_nodes * kB, s) != cudaSuccess ||
      cudaMemsetAsync(d.alive, 1, (size_t) nb_nodes, s) != cudaSuccess)
    return TRN_ERR_CUDA;

  const int gv = grid_for(nb_nodes), ge = grid_for(nb_elems);
  k_na_expand<<<ge, TRN_THREADS, 0, s>>>(d_tris, nb_elems, nb_nodes, d.tri, d.err);
  k_na_points<<<gv, TRN_THREADS, 0, s>>>(d_points, nb_nodes, d.pts);
  k_fill_stencils<<<ge, TRN_THREADS, 0, s>>>(d, nb_elems);
  k_sort_stencils<<<gv, TRN_THREADS, 0, s>>>(d, nb_nodes);
  k_build_vicin<<<gv, TRN_THREADS, 0, s>>>(d, nb_nodes, 0);

  const double target = (double) (int) std::floor(nb_nodes * target_factor);
  const double scale_exp = lp_norm ? -1. / (2 * lp_norm + 2) : 0.5;
  const double eig_min = 1 / trn_pow(h_min, 2);
  const double eig_max = 1 / trn_pow(h_max, 2);
  k_gradient<<<gv, TRN_THREADS, 0, s>>>(d, nb_nodes, d_solut, grad, nullptr);
  k_hessian_local<<<gv, TRN_THREADS, 0, s>>>(d, nb_nodes, grad, scale_exp, nullptr, nullptr);
  k_complexity_term<<<ge, TRN_THREADS, 0, s>>>(d, nb_elems, terms);
  k_sum_partial<<<ge, TRN_THREADS, 0, s>>>(terms, nb_elems, terms + kMaxE);
  k_sum_final<<<1, TRN_THREADS, 0, s>>>(terms + kMaxE, ge, cplx);
  k_normalize<<<gv, TRN_THREADS, 0, s>>>(d, nb_nodes, cplx, target, eig_min, eig_max);
  k_na_tensor<<<gv, TRN_THREADS, 0, s>>>(d.ten, nb_nodes, d_tensor);
  if (cudaPeekAtLastError() != cudaSuccess) return TRN_ERR_CUDA;

  int err = 0;
  if (cudaMemcpyAsync(&err, d.err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TRN_ERR_CUDA;
  if (err == TRN_DERR_CAPACITY || err == TRN_DERR_BUCKET) {
    std::fprintf(stderr, "trn_metric_noalloc: a vertex has more than %d incident triangles\n",
                 TRN_NOALLOC_BUCKET);
    return TRN_ERR_CAPACITY;
  }
  if (err) return TRN_ERR_INVALID;
  return TRN_OK;
}
