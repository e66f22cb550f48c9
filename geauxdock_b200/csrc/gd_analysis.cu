// gd_analysis.cu -- post-analysis of a docking job's replicas: each replica's
// best pose (the lowest total energy it visited, kept by the Monte Carlo
// kernel in its FP64 statistics), its RMSD to a reference pose, and the best
// poses clustered in order of energy with an RMSD cut-off.  The reference
// records poses (src/common/geauxdock.h:374-378) and sketches a medoid
// summary with cluster size, relative size, z-score and mean energy
// (src/analysis/record.h:50-59) that it never fills; this is that summary.
//
// Clustering (leader, in energy order): a pose joins the first cluster whose
// leader is within the cut-off, else it leads a new one.  It runs as rounds in
// one CTA: the lowest-energy unassigned pose leads the next cluster and every
// unassigned pose within the cut-off of it joins, which assigns each pose to
// the same cluster as the sequential rule.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "gd_internal.h"
#include "gd_pack.h"
#include "gdock.h"

namespace gd {
namespace {

// Ligand coordinates of the best pose of replica order[i] (the transform of the
// energy routine, kernel_cuda_l1_montecarlo.cu:336-380), one thread per atom.
__global__ void best_pose_kernel(const DevJob *jobp, const int *order, int n, int lstride, float4 *out)
{
  const DevJob &J = *jobp;
  const int i = blockIdx.x;
  if (i >= n) return;
  const int r = order[i];
  __shared__ float mm[6];
  __shared__ int ilig;
  if (threadIdx.x < 6) mm[threadIdx.x] = J.stats[r].best_mm[threadIdx.x];
  if (threadIdx.x == 0) ilig = J.rep[r].idx_lig;
  __syncthreads();
  float s1, c1, s2, c2, s3, c3;
  sincosf(mm[3], &s1, &c1);
  sincosf(mm[4], &s2, &c2);
  sincosf(mm[5], &s3, &c3);
  const float r00 = c1 * c2, r01 = c1 * s2 * s3 - c3 * s1, r02 = s1 * s3 + c1 * c3 * s2;
  const float r10 = c2 * s1, r11 = c1 * c3 + s1 * s2 * s3, r12 = c3 * s1 * s2 - c1 * s3;
  const float r20 = -s2, r21 = c2 * s3, r22 = c2 * c3;
  const float *lc = J.lcenter + 3 * ilig;
  const float tx = mm[0] + lc[0], ty = mm[1] + lc[1], tz = mm[2] + lc[2];
  for (int a = threadIdx.x; a < J.natom; a += blockDim.x) {
    const float4 v = J.lig[(size_t)ilig * J.lstride + a];
    out[(size_t)i * lstride + a] = make_float4(r00 * v.x + r01 * v.y + r02 * v.z + tx,
                                               r10 * v.x + r11 * v.y + r12 * v.z + ty,
                                               r20 * v.x + r21 * v.y + r22 * v.z + tz, 0.f);
  }
}

// RMSD of every best pose to the reference pose (coordinates ref[L]).
__global__ void ref_rmsd_kernel(const float4 *pose, const float4 *ref, int n, int L, int lstride, float *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int a = 0; a < L; ++a) {
    const float4 p = pose[(size_t)i * lstride + a], q = ref[a];
    const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
    s = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, s)));
  }
  out[i] = sqrtf(s / (float)L);
}

// Leader clustering of poses already in energy order, one CTA.  assign[i]:
// cluster of pose i, in order of creation; *ncl: clusters.
__global__ void leader_cluster_kernel(const float4 *pose, int n, int L, int lstride, float cut2L, int *assign,
                                      int *ncl)
{
  extern __shared__ float4 lead[];  // [L] leader coordinates
  __shared__ int s_next;
  for (int i = threadIdx.x; i < n; i += blockDim.x) assign[i] = -1;
  __syncthreads();
  int c = 0, from = 0;
  for (;;) {
    if (threadIdx.x == 0) s_next = n;
    __syncthreads();
    for (int i = from + threadIdx.x; i < n; i += blockDim.x)
      if (assign[i] < 0) atomicMin(&s_next, i);
    __syncthreads();
    const int l = s_next;
    if (l >= n) break;  // every pose assigned (uniform: all threads read s_next)
    for (int a = threadIdx.x; a < L; a += blockDim.x) lead[a] = pose[(size_t)l * lstride + a];
    __syncthreads();
    for (int i = l + threadIdx.x; i < n; i += blockDim.x) {
      if (assign[i] >= 0) continue;
      float s = 0.f;
      for (int a = 0; a < L; ++a) {
        const float4 p = pose[(size_t)i * lstride + a], q = lead[a];
        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        s = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, s)));
      }
      if (i == l || s <= cut2L) assign[i] = c;
    }
    __syncthreads();
    ++c;
    from = l + 1;
  }
  if (threadIdx.x == 0) *ncl = c;
}

}  // namespace

int cluster_job(const DevJob &J, const DevJob *d_job, cudaStream_t st, int ref_lig, const float ref_mm[6],
                float rmsd_cut, gd_cluster_t *clusters, int max_clusters, int *n_clusters, int *cluster_of,
                float *rmsd_to_ref)
{
  const int n = J.nrep, L = J.natom, ls = J.lstride;
  if (n < 1) return fail(GD_E_INVALID, "no replicas");
  if (ref_lig < 0 || ref_lig >= J.nlig) return fail(GD_E_INVALID, "reference ligand conformation %d", ref_lig);
  if (!(rmsd_cut >= 0.f)) return fail(GD_E_INVALID, "rmsd_cut = %g", (double)rmsd_cut);
  std::vector<RepStats> st_h(n);
  GD_CUDA(cudaMemcpyAsync(st_h.data(), J.stats, sizeof(RepStats) * n, cudaMemcpyDeviceToHost, st));
  GD_CUDA(cudaStreamSynchronize(st));
  for (int r = 0; r < n; ++r)
    if (st_h[r].best_step < 0) return fail(GD_E_STATE, "replica %d has no evaluated pose (run the ensemble first)", r);
  // energy order (ties by replica index)
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return st_h[a].best_e < st_h[b].best_e; });

  // the reference pose as one more "replica": the ligand conformation at ref_mm
  int *d_order = nullptr, *d_assign = nullptr, *d_ncl = nullptr;
  float4 *d_pose = nullptr, *d_ref = nullptr;
  float *d_rmsd = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_order);
    cudaFree(d_assign);
    cudaFree(d_ncl);
    cudaFree(d_pose);
    cudaFree(d_ref);
    cudaFree(d_rmsd);
  };
#define AN_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t ce_ = (call);                                                                  \
    if (ce_ != cudaSuccess) {                                                                  \
      cleanup();                                                                               \
      return fail(GD_E_CUDA, "cluster analysis: %s: %s", #call, cudaGetErrorString(ce_));      \
    }                                                                                          \
  } while (0)
  AN_CUDA(cudaMalloc(&d_order, sizeof(int) * n));
  AN_CUDA(cudaMalloc(&d_assign, sizeof(int) * n));
  AN_CUDA(cudaMalloc(&d_ncl, sizeof(int)));
  AN_CUDA(cudaMalloc(&d_pose, sizeof(float4) * (size_t)n * ls));
  AN_CUDA(cudaMalloc(&d_ref, sizeof(float4) * (size_t)ls));
  AN_CUDA(cudaMalloc(&d_rmsd, sizeof(float) * n));
  AN_CUDA(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  best_pose_kernel<<<n, 64, 0, st>>>(d_job, d_order, n, ls, d_pose);
  AN_CUDA(cudaGetLastError());
  {
    // reference coordinates on the host, the same transform in FP32
    std::vector<float4> lig(ls), ref(ls);
    std::vector<float> lc(3);
    AN_CUDA(cudaMemcpyAsync(lig.data(), J.lig + (size_t)ref_lig * ls, sizeof(float4) * ls, cudaMemcpyDeviceToHost, st));
    AN_CUDA(cudaMemcpyAsync(lc.data(), J.lcenter + 3 * ref_lig, sizeof(float) * 3, cudaMemcpyDeviceToHost, st));
    AN_CUDA(cudaStreamSynchronize(st));
    const float *m = ref_mm;
    const float zero[6] = {0, 0, 0, 0, 0, 0};
    if (!m) m = zero;
    const float s1 = std::sin(m[3]), c1 = std::cos(m[3]), s2 = std::sin(m[4]), c2 = std::cos(m[4]),
                s3 = std::sin(m[5]), c3 = std::cos(m[5]);
    const float R[3][3] = {{c1 * c2, c1 * s2 * s3 - c3 * s1, s1 * s3 + c1 * c3 * s2},
                           {c2 * s1, c1 * c3 + s1 * s2 * s3, c3 * s1 * s2 - c1 * s3},
                           {-s2, c2 * s3, c2 * c3}};
    for (int a = 0; a < L; ++a) {
      const float4 v = lig[a];
      ref[a] = make_float4(R[0][0] * v.x + R[0][1] * v.y + R[0][2] * v.z + m[0] + lc[0],
                           R[1][0] * v.x + R[1][1] * v.y + R[1][2] * v.z + m[1] + lc[1],
                           R[2][0] * v.x + R[2][1] * v.y + R[2][2] * v.z + m[2] + lc[2], 0.f);
    }
    AN_CUDA(cudaMemcpyAsync(d_ref, ref.data(), sizeof(float4) * ls, cudaMemcpyHostToDevice, st));
    AN_CUDA(cudaStreamSynchronize(st));
  }
  ref_rmsd_kernel<<<(n + 127) / 128, 128, 0, st>>>(d_pose, d_ref, n, L, ls, d_rmsd);
  AN_CUDA(cudaGetLastError());
  leader_cluster_kernel<<<1, 1024, sizeof(float4) * ls, st>>>(d_pose, n, L, ls, rmsd_cut * rmsd_cut * (float)L,
                                                               d_assign, d_ncl);
  AN_CUDA(cudaGetLastError());
  std::vector<int> assign(n);
  std::vector<float> rmsd(n);
  int ncl = 0;
  AN_CUDA(cudaMemcpyAsync(assign.data(), d_assign, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  AN_CUDA(cudaMemcpyAsync(rmsd.data(), d_rmsd, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  AN_CUDA(cudaMemcpyAsync(&ncl, d_ncl, sizeof(int), cudaMemcpyDeviceToHost, st));
  AN_CUDA(cudaStreamSynchronize(st));
#undef AN_CUDA
  cleanup();

  // cluster summaries; z-score of a leader's energy against all best energies
  double mean = 0, var = 0;
  for (int r = 0; r < n; ++r) mean += st_h[r].best_e;
  mean /= n;
  for (int r = 0; r < n; ++r) var += (st_h[r].best_e - mean) * (st_h[r].best_e - mean);
  const double sd = std::sqrt(var / n);
  std::vector<gd_cluster_t> cl(ncl);
  std::vector<double> esum(ncl, 0.0);
  for (int c = 0; c < ncl; ++c) {
    std::memset(&cl[c], 0, sizeof(gd_cluster_t));
    cl[c].representative = -1;
  }
  for (int i = 0; i < n; ++i) {
    const int c = assign[i], r = order[i];
    if (c < 0 || c >= ncl) return fail(GD_E_CUDA, "cluster analysis: pose %d unassigned", i);
    if (cl[c].representative < 0) {
      cl[c].representative = r;
      cl[c].rep_energy = (float)st_h[r].best_e;
      cl[c].rep_rmsd = rmsd[i];
      cl[c].z_score = sd > 0 ? (float)((st_h[r].best_e - mean) / sd) : 0.f;
    }
    cl[c].size += 1;
    esum[c] += st_h[r].best_e;
    if (cluster_of) cluster_of[r] = c;
    if (rmsd_to_ref) rmsd_to_ref[r] = rmsd[i];
  }
  for (int c = 0; c < ncl; ++c) {
    cl[c].mean_energy = (float)(esum[c] / cl[c].size);
    cl[c].relative_size = (float)cl[c].size / (float)n;
  }
  for (int c = 0; c < ncl && c < max_clusters; ++c) clusters[c] = cl[c];
  *n_clusters = ncl;
  return GD_OK;
}

}  // namespace gd
