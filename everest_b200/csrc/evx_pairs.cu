// Pair index: for every static edge (u, v) the run of its temporal edges
// {eid, t}, ascending in eid, plus an open-addressing hash table
// (u, v) -> (start, len).  It lets the search count a closing last motif
// edge by range arithmetic (the number of u->v edges with id after the
// previous edge and t <= t(e_0) + delta) instead of scanning a list.
//
// Built on the device from the packed edge array: a stable 64-bit radix sort
// of (u, v) keys with edge-id values (CUB), run-length encoding of the sorted
// keys, and a parallel hash insert (atomicCAS on the 64-bit key).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>

#include "evx_internal.cuh"

namespace evx {
namespace {

__global__ void pair_keys_kernel(const int4 *__restrict__ edges, unsigned long long *__restrict__ keys,
                                 int *__restrict__ vals, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int4 e = edges[i];
    keys[i] = pair_key(e.x, e.y);
    vals[i] = i;
  }
}

__global__ void pair_rec_kernel(const int *__restrict__ eids, const int4 *__restrict__ edges,
                                int2 *__restrict__ rec, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e = eids[i];
    rec[i] = make_int2(e, edges[e].z);
  }
}

// pair_loc[e] = {position of e in pair_rec, end of its run}
__global__ void pair_loc_kernel(const int *__restrict__ eids, const int *__restrict__ starts,
                                const int *__restrict__ lens, const int *__restrict__ num_runs,
                                int2 *__restrict__ loc) {
  const int P = *num_runs;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < P; r += gridDim.x * blockDim.x) {
    const int b = starts[r], e = b + lens[r];
    for (int i = b; i < e; i++) loc[eids[i]] = make_int2(i, e);
  }
}

// dir[r] = {v, start} of run r (runs sorted by (u, v)); dir[P] = sentinel;
// node_cnt[u] = runs of source u
__global__ void pair_dir_kernel(const unsigned long long *__restrict__ ukeys,
                                const int *__restrict__ starts, const int *__restrict__ num_runs,
                                int2 *__restrict__ dir, int *__restrict__ node_cnt, int n_edges) {
  const int P = *num_runs;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= P; r += gridDim.x * blockDim.x) {
    if (r == P) {
      dir[r] = make_int2(0x7fffffff, n_edges);
    } else {
      const unsigned long long k = ukeys[r];
      dir[r] = make_int2((int)(unsigned)(k & 0xffffffffull), starts[r]);
      atomicAdd(node_cnt + (int)(k >> 32), 1);
    }
  }
}

// rev[e] for e = (u, v): the entries of the reverse pair's run (v, u) after
// e (edge id greater than e), as {first such position, end of the run};
// {0, 0} when there is no v -> u edge.
__global__ void rev_loc_kernel(const GraphView g, int2 *__restrict__ rev, int n) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int4 ed = g.edges[e];
    const int2 f = pair_find(g, ed.y, ed.x);
    int lo = f.x, hi = f.x + f.y;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (g.pair_rec[mid].x > e) hi = mid; else lo = mid + 1;
    }
    rev[e] = f.y > 0 ? make_int2(lo, f.x + f.y) : make_int2(0, 0);
  }
}

// Cross-list starts: for e = (u, v), the first position of out(v) and of
// in(u) whose edge comes after e (the two endpoint lists e is not in), so
// a search that extends e from either endpoint starts without a binary
// search.
__global__ void cross_pos_kernel(const int4 *__restrict__ edges, const int4 *__restrict__ node_rng,
                                 const int4 *__restrict__ out_rec, const int4 *__restrict__ in_rec,
                                 int *__restrict__ cross_out, int *__restrict__ cross_in, int n) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int4 ed = edges[e];
    int lo = node_rng[ed.y].x, hi = node_rng[ed.y].y;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (out_rec[mid].x > e) hi = mid; else lo = mid + 1;
    }
    cross_out[e] = lo;
    lo = node_rng[ed.x].z; hi = node_rng[ed.x].w;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (in_rec[mid].x > e) hi = mid; else lo = mid + 1;
    }
    cross_in[e] = lo;
  }
}

// Mark each adjacency record whose edge is followed by another entry of its
// pair run (top bit of the record's fourth word) and whose reverse pair has
// an entry after it (kRevLater).
__global__ void mark_runs_kernel(int4 *__restrict__ out_rec, int4 *__restrict__ in_rec,
                                 const int2 *__restrict__ loc, const int2 *__restrict__ rev, int n) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int eo = out_rec[p].x, ei = in_rec[p].x;
    const int2 lo = loc[eo], li = loc[ei];
    int fo = lo.x + 1 < lo.y ? (int)0x80000000u : 0;
    int fi = li.x + 1 < li.y ? (int)0x80000000u : 0;
    const int2 ro = rev[eo], ri = rev[ei];
    if (ro.x < ro.y) fo |= kRevLater;
    if (ri.x < ri.y) fi |= kRevLater;
    out_rec[p].w |= fo;
    in_rec[p].w |= fi;
  }
}

// Neighbour signatures: one bit per neighbour (sig_bit) in each endpoint's word.
__global__ void pair_sig_kernel(const int4 *__restrict__ edges, unsigned long long *__restrict__ sig_out,
                                unsigned long long *__restrict__ sig_in, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int4 e = edges[i];
    atomicOr(sig_out + e.x, 1ull << sig_bit(e.y));
    atomicOr(sig_in + e.y, 1ull << sig_bit(e.x));
  }
}

__global__ void pair_clear_kernel(int4 *__restrict__ tab, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    tab[i] = make_int4(-1, -1, 0, 0);
}

// Insert every run; the probe sequence is bounded by the table size, and the
// longest probe actually used is recorded so lookups can stop there.
__global__ void pair_insert_kernel(const unsigned long long *__restrict__ ukeys,
                                   const int *__restrict__ starts, const int *__restrict__ lens,
                                   const int *__restrict__ num_runs, int4 *__restrict__ tab,
                                   unsigned long long mask, int *__restrict__ max_probe,
                                   int *__restrict__ overflow) {
  const int P = *num_runs;
  int longest = 0;  // this thread's longest probe; one atomicMax per warp at the end
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const unsigned long long key = ukeys[p];
    unsigned long long h = pair_hash(key) & mask;
    bool done = false;
    for (unsigned long long i = 0; i <= mask; i++) {
      unsigned long long *slot = reinterpret_cast<unsigned long long *>(tab + h);
      const unsigned long long prev = atomicCAS(slot, ~0ull, key);
      if (prev == ~0ull) {
        tab[h].z = starts[p];
        tab[h].w = lens[p];
        longest = max(longest, (int)i + 1);
        done = true;
        break;
      }
      h = (h + 1) & mask;
    }
    if (!done) atomicExch(overflow, 1);
  }
  longest = __reduce_max_sync(0xffffffffu, (unsigned)longest);
  if ((threadIdx.x & 31) == 0 && longest > 0) atomicMax(max_probe, longest);
}

}  // namespace

int build_pair_index(DeviceGraph &g, cudaStream_t s) {
  const int64_t E = g.num_edges;
  {
    const size_t vs = (size_t)(g.num_vertices > 0 ? g.num_vertices : 1);
    EVX_CUDA(dev_alloc((void **)&g.sig_out, sizeof(unsigned long long) * vs, g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.sig_in, sizeof(unsigned long long) * vs, g.device, s));
    EVX_CUDA(cudaMemsetAsync(g.sig_out, 0, sizeof(unsigned long long) * vs, s));
    EVX_CUDA(cudaMemsetAsync(g.sig_in, 0, sizeof(unsigned long long) * vs, s));
    g.bytes += (int64_t)(2 * sizeof(unsigned long long) * vs);
  }
  if (E <= 0) {
    g.pair_mask = 0;
    g.pair_max_probe = 0;
    EVX_CUDA(dev_alloc((void **)&g.pair_tab, sizeof(int4), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.pair_rec, sizeof(int2), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.pair_loc, sizeof(int2), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.rev_loc, sizeof(int2), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.cross_out, sizeof(int), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.cross_in, sizeof(int), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.pair_dir, sizeof(int2), g.device, s));
    EVX_CUDA(dev_alloc((void **)&g.dir_off, sizeof(int) * (size_t)(g.num_vertices + 1), g.device, s));
    EVX_CUDA(cudaMemsetAsync(g.pair_tab, 0xff, sizeof(int4), s));
    EVX_CUDA(cudaMemsetAsync(g.dir_off, 0, sizeof(int) * (size_t)(g.num_vertices + 1), s));
    {
      const int2 sentinel = make_int2(0x7fffffff, 0);
      EVX_CUDA(cudaMemcpyAsync(g.pair_dir, &sentinel, sizeof(int2), cudaMemcpyHostToDevice, s));
      EVX_CUDA(cudaStreamSynchronize(s));
    }
    g.bytes += sizeof(int4) + 5 * sizeof(int2) + sizeof(int) * (g.num_vertices + 1);
    return EVX_OK;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
  const int grid = sms * 8, block = 256;
  const int n = (int)E;
  unsigned long long *keys = nullptr, *keys_sorted = nullptr, *ukeys = nullptr;
  int *vals = nullptr, *vals_sorted = nullptr, *lens = nullptr, *starts = nullptr, *ctr = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0, t1 = 0, t2 = 0, t3 = 0;
  int rc = EVX_OK;
  auto A = [&](void **p, size_t b) {
    if (rc == EVX_OK) {
      cudaError_t e = dev_alloc(p, b, g.device, s);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMallocAsync(pair index scratch)");
    }
  };
  A((void **)&keys, sizeof(unsigned long long) * n);
  A((void **)&keys_sorted, sizeof(unsigned long long) * n);
  A((void **)&ukeys, sizeof(unsigned long long) * n);
  A((void **)&vals, sizeof(int) * n);
  A((void **)&vals_sorted, sizeof(int) * n);
  A((void **)&lens, sizeof(int) * n);
  A((void **)&starts, sizeof(int) * n);
  A((void **)&ctr, sizeof(int) * 4);  // [0] runs, [1] max probe, [2] overflow
  if (rc) goto cleanup;
  // key bits actually used: u and v < V
  {
    int vb = 1;
    while ((1ll << vb) < g.num_vertices + 1 && vb < 31) vb++;
    const int end_bit = 32 + vb;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, keys, keys_sorted, vals, vals_sorted, n, 0, end_bit, s);
    cub::DeviceRunLengthEncode::Encode(nullptr, t2, keys_sorted, ukeys, lens, ctr, n, s);
    cub::DeviceScan::ExclusiveSum(nullptr, t3, lens, starts, n, s);
    tmp_bytes = t1 > t2 ? t1 : t2;
    tmp_bytes = tmp_bytes > t3 ? tmp_bytes : t3;
    A(&tmp, tmp_bytes);
    if (rc) goto cleanup;
    EVX_CUDA(cudaMemsetAsync(lens, 0, sizeof(int) * n, s));
    pair_keys_kernel<<<grid, block, 0, s>>>(g.edges, keys, vals, n);
    pair_sig_kernel<<<grid, block, 0, s>>>(g.edges, g.sig_out, g.sig_in, n);
    cub::DeviceRadixSort::SortPairs(tmp, t1, keys, keys_sorted, vals, vals_sorted, n, 0, end_bit, s);
    cub::DeviceRunLengthEncode::Encode(tmp, t2, keys_sorted, ukeys, lens, ctr, n, s);
    // lens beyond the run count are never read by the scan's consumers; the
    // scan runs over n entries and only the first 'runs' starts are used
    cub::DeviceScan::ExclusiveSum(tmp, t3, lens, starts, n, s);
  }
  {
    int runs = 0;
    EVX_CUDA(cudaMemcpyAsync(&runs, ctr, sizeof(int), cudaMemcpyDeviceToHost, s));
    EVX_CUDA(cudaStreamSynchronize(s));
    long long cap = 1;
    while (cap < 2ll * runs + 2) cap <<= 1;
    g.pair_mask = (unsigned long long)(cap - 1);
    cudaError_t e = dev_alloc((void **)&g.pair_tab, sizeof(int4) * (size_t)cap, g.device, s);
    if (e == cudaSuccess) e = dev_alloc((void **)&g.pair_rec, sizeof(int2) * (size_t)n, g.device, s);
    if (e == cudaSuccess) e = dev_alloc((void **)&g.pair_loc, sizeof(int2) * (size_t)n, g.device, s);
    if (e == cudaSuccess) e = dev_alloc((void **)&g.rev_loc, sizeof(int2) * (size_t)n, g.device, s);
    if (e == cudaSuccess) e = dev_alloc((void **)&g.cross_out, sizeof(int) * (size_t)n, g.device, s);
    if (e == cudaSuccess) e = dev_alloc((void **)&g.cross_in, sizeof(int) * (size_t)n, g.device, s);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMalloc(pair index)"); goto cleanup; }
    g.bytes += (int64_t)(sizeof(int4) * cap + 4 * sizeof(int2) * n);
    EVX_CUDA(cudaMemsetAsync(ctr + 1, 0, 2 * sizeof(int), s));
    pair_clear_kernel<<<grid, block, 0, s>>>(g.pair_tab, cap);
    pair_rec_kernel<<<grid, block, 0, s>>>(vals_sorted, g.edges, g.pair_rec, n);
    pair_loc_kernel<<<grid, block, 0, s>>>(vals_sorted, starts, lens, ctr, g.pair_loc);
    pair_insert_kernel<<<grid, block, 0, s>>>(ukeys, starts, lens, ctr, g.pair_tab, g.pair_mask, ctr + 1,
                                              ctr + 2);
    // per-node directory of distinct out-neighbours (sorted) -> pair runs
    {
      const int64_t V = g.num_vertices;
      cudaError_t e2 = dev_alloc((void **)&g.pair_dir, sizeof(int2) * ((size_t)runs + 1), g.device, s);
      if (e2 == cudaSuccess) e2 = dev_alloc((void **)&g.dir_off, sizeof(int) * (size_t)(V + 1), g.device, s);
      if (e2 != cudaSuccess) { rc = cuda_fail(e2, "cudaMalloc(pair directory)"); goto cleanup; }
      g.bytes += (int64_t)(sizeof(int2) * ((size_t)runs + 1) + sizeof(int) * (V + 1));
      int *node_cnt = nullptr;
      A((void **)&node_cnt, sizeof(int) * (size_t)(V + 1));
      if (rc) goto cleanup;
      EVX_CUDA(cudaMemsetAsync(node_cnt, 0, sizeof(int) * (size_t)(V + 1), s));
      pair_dir_kernel<<<grid, block, 0, s>>>(ukeys, starts, ctr, g.pair_dir, node_cnt, n);
      size_t t4 = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, t4, node_cnt, g.dir_off, (int)(V + 1), s);
      if (t4 > tmp_bytes) {
        dev_free(tmp, s);
        tmp = nullptr;
        A(&tmp, t4);
        if (rc) goto cleanup;
        tmp_bytes = t4;
      }
      cub::DeviceScan::ExclusiveSum(tmp, t4, node_cnt, g.dir_off, (int)(V + 1), s);
      dev_free(node_cnt, s);
    }
    int h[2] = {0, 0};
    EVX_CUDA(cudaGetLastError());
    EVX_CUDA(cudaMemcpyAsync(h, ctr + 1, sizeof(h), cudaMemcpyDeviceToHost, s));
    EVX_CUDA(cudaStreamSynchronize(s));
    if (h[1]) { rc = fail(EVX_ERR_CUDA, "pair index insert overflow"); goto cleanup; }
    g.pair_max_probe = h[0];
    rev_loc_kernel<<<grid, block, 0, s>>>(g.view(), g.rev_loc, n);
    cross_pos_kernel<<<grid, block, 0, s>>>(g.edges, g.node_rng, g.out_rec, g.in_rec, g.cross_out, g.cross_in, n);
    mark_runs_kernel<<<grid, block, 0, s>>>(g.out_rec, g.in_rec, g.pair_loc, g.rev_loc, n);
    EVX_CUDA(cudaGetLastError());
  }
cleanup:
  dev_free(keys, s);
  dev_free(keys_sorted, s);
  dev_free(ukeys, s);
  dev_free(vals, s);
  dev_free(vals_sorted, s);
  dev_free(lens, s);
  dev_free(starts, s);
  dev_free(ctr, s);
  dev_free(tmp, s);
  if (rc == EVX_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_fail(e, "pair index build");
  }
  return rc;
}

}  // namespace evx
