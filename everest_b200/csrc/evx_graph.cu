// Device graph: upload of the host graph arrays and on-device packing into
// the 16-byte record layout the search kernels read.
//
// Host-format inputs are the reference's HostGraphData arrays
// (include/data.h:174-186): Eg (AoS {u,v,t}), outEdgesV / inEdgesV (edge ids
// grouped by endpoint, ascending), outEdgesR / inEdgesR (CSR offsets) and
// Euid.  The upload moves exactly those bytes (24 E + 8 (V+1), as
// calcTotalBytes, src/core/gpu/data.cu:22-24) and expands them on the device
// into the layout described in evx_internal.cuh (16-byte adjacency records
// carrying each edge's position in its other list, per-node int4 ranges).
#include <climits>

#include "evx_internal.cuh"

namespace evx {
namespace {

// positions: outpos[out_v[p]] = p, inpos[in_v[p]] = p
__global__ void scatter_pos_kernel(const int *__restrict__ out_v, const int *__restrict__ in_v,
                                   int *__restrict__ outpos, int *__restrict__ inpos, int n) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    outpos[out_v[p]] = p;
    inpos[in_v[p]] = p;
  }
}

__global__ void pack_edges_kernel(const int *__restrict__ eg, const int *__restrict__ euid_in,
                                  const int *__restrict__ outpos, int4 *__restrict__ edges,
                                  int *__restrict__ euid, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    edges[i] = make_int4(eg[3 * i], eg[3 * i + 1], eg[3 * i + 2], outpos[i]);
    euid[i] = euid_in ? euid_in[i] : i;
  }
}

__global__ void pack_rec_kernel(const int *__restrict__ out_v, const int *__restrict__ in_v,
                                const int4 *__restrict__ edges, const int *__restrict__ inpos,
                                int4 *__restrict__ out_rec, int4 *__restrict__ in_rec, int n) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int eo = out_v[p];
    const int4 a = edges[eo];
    out_rec[p] = make_int4(eo, a.y, a.z, inpos[eo]);
    const int ei = in_v[p];
    const int4 b = edges[ei];
    in_rec[p] = make_int4(ei, b.x, b.z, b.w);
  }
}

__global__ void pack_nodes_kernel(const int *__restrict__ out_r, const int *__restrict__ in_r,
                                  int4 *__restrict__ node_rng, int nv) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nv; x += gridDim.x * blockDim.x) {
    node_rng[x] = make_int4(out_r[x], out_r[x + 1], in_r[x], in_r[x + 1]);
  }
}

// Input checks: edge ids in [0, E), vertex ids in [0, V), timestamps sorted,
// CSR offsets monotone from 0 to E.  Bits of *err name the failed check.
__global__ void validate_kernel(const int *__restrict__ eg, const int *__restrict__ out_v,
                                const int *__restrict__ in_v, const int *__restrict__ out_r,
                                const int *__restrict__ in_r, int E, int V, int *err) {
  const int n = max(E, V + 1);
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < E) {
      if ((unsigned)out_v[i] >= (unsigned)E || (unsigned)in_v[i] >= (unsigned)E) bad |= 1;
      if ((unsigned)eg[3 * i] >= (unsigned)V || (unsigned)eg[3 * i + 1] >= (unsigned)V) bad |= 2;
      if (i > 0 && eg[3 * i + 2] < eg[3 * i - 1]) bad |= 4;
    }
    if (i < V && (out_r[i + 1] < out_r[i] || in_r[i + 1] < in_r[i])) bad |= 8;
    if (i == 0 && (out_r[0] != 0 || in_r[0] != 0 || out_r[V] != E || in_r[V] != E)) bad |= 16;
  }
  if (bad) atomicOr(err, bad);
}

// min / max timestamp (for the t + delta overflow check)
__global__ void t_range_kernel(const int4 *__restrict__ edges, int n, int *out) {
  int lo = INT_MAX, hi = INT_MIN;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int t = edges[i].z;
    lo = min(lo, t);
    hi = max(hi, t);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, lo);
    atomicMax(out + 1, hi);
  }
}

__global__ void t_range_init_kernel(int *out) {
  out[0] = INT_MAX;
  out[1] = INT_MIN;
}

}  // namespace

int pack_graph(DeviceGraph &g, const int *eg_d, const int *out_v_d, const int *in_v_d,
               const int *out_r_d, const int *in_r_d, const int *euid_d, cudaStream_t s) {
  const int64_t E = g.num_edges, V = g.num_vertices;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
  const int grid = sms * 8, block = 256;
  if (V > 0) pack_nodes_kernel<<<grid, block, 0, s>>>(out_r_d, in_r_d, g.node_rng, (int)V);
  if (E > 0) {
    int *outpos = nullptr;  // edges[].w, staged
    EVX_CUDA(dev_alloc((void **)&outpos, sizeof(int) * (size_t)E, g.device, s));
    scatter_pos_kernel<<<grid, block, 0, s>>>(out_v_d, in_v_d, outpos, g.inpos, (int)E);
    pack_edges_kernel<<<grid, block, 0, s>>>(eg_d, euid_d, outpos, g.edges, g.euid, (int)E);
    pack_rec_kernel<<<grid, block, 0, s>>>(out_v_d, in_v_d, g.edges, g.inpos, g.out_rec, g.in_rec,
                                           (int)E);
    dev_free(outpos, s);
  }
  EVX_CUDA(cudaGetLastError());
  return EVX_OK;
}

int validate_graph(int device, int64_t E, int64_t V, const int *eg_d, const int *out_v_d, const int *in_v_d,
                   const int *out_r_d, const int *in_r_d, cudaStream_t s) {
  int *err = nullptr;
  EVX_CUDA(dev_alloc((void **)&err, sizeof(int), device, s));
  EVX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  validate_kernel<<<sms * 8, 256, 0, s>>>(eg_d, out_v_d, in_v_d, out_r_d, in_r_d, (int)E, (int)V, err);
  int h = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dev_free(err, s);
  if (e != cudaSuccess) return cuda_fail(e, "graph validation");
  if (h & 1) return fail(EVX_ERR_INVALID, "edge id out of range in out/in lists");
  if (h & 2) return fail(EVX_ERR_INVALID, "vertex id out of range in Eg");
  if (h & 4) return fail(EVX_ERR_INVALID, "edges are not sorted by timestamp");
  if (h & 8) return fail(EVX_ERR_INVALID, "CSR offsets are not monotone");
  if (h & 16) return fail(EVX_ERR_INVALID, "CSR offsets must start at 0 and end at num_edges");
  return EVX_OK;
}

int graph_t_range(DeviceGraph &g, int *scratch_d, cudaStream_t s) {
  int h[2] = {0, 0};
  t_range_init_kernel<<<1, 1, 0, s>>>(scratch_d);
  if (g.num_edges > 0) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
    t_range_kernel<<<sms * 4, 256, 0, s>>>(g.edges, (int)g.num_edges, scratch_d);
  }
  EVX_CUDA(cudaGetLastError());
  EVX_CUDA(cudaMemcpyAsync(h, scratch_d, sizeof(h), cudaMemcpyDeviceToHost, s));
  EVX_CUDA(cudaStreamSynchronize(s));
  g.min_t = g.num_edges ? h[0] : 0;
  g.max_t = g.num_edges ? h[1] : 0;
  return EVX_OK;
}

}  // namespace evx
