// CSR pattern of the reduced free/free system, built on the device.
//
// The reference accumulates (row, col) keys into an unordered_map element by element
// (src/fem/assembly.cpp:76-100) and flushes unordered COO triplets (211-221). Here the
// pattern is built once per mesh and DOF map, in canonical sorted CSR form:
//   1. every element emits the n^2 node-pair keys a*N + b; a device radix sort and
//      unique give the node adjacency graph, sorted by (a, b);
//   2. each node a gets its free-component mask; all rows of a share one column
//      structure (the free components of a's neighbours, ascending), so per node
//      rowlen(a) = sum over neighbours of their free-component count and the offset
//      of neighbour b inside a's rows is the running sum before b;
//   3. node_base(a) = exclusive scan of (free rows of a) * rowlen(a); row_ptr and
//      col_idx follow. This relies on the reference's free numbering being ascending
//      in g = 3*node + comp (constraint_transform.cpp:78-82), which is validated;
//   4. the slot map stores, per element and ordered node pair (a, b), the position of b
//      in a's adjacency list (uint16), so the row gather adds block (a, b) into a's
//      rows with no search; the gather keeps the list length of every node (adj_len)
//      and, for the nodes with a neighbour that is not fully free (their rows are
//      compressed), the neighbours themselves (bnd_ptr, bnd_node).
// The pattern is topological: an entry whose every element contribution is exactly
// zero is kept (the reference skips exact-zero contributions, assembly.cpp:90).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "cxg_internal.cuh"

namespace cxg {
namespace {

__global__ void check_conn_kernel(const int32_t* conn, int64_t total, int64_t n_nodes, int* flag,
                                  unsigned long long* bad, int npe) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t v = conn[i];
    if (v < 0 || v >= n_nodes) {
      atomicExch(flag, 1);
      atomicMin(bad, static_cast<unsigned long long>(i / npe));
    }
  }
}

__global__ void free_flags_kernel(const int32_t* dof_eq, int64_t ndof, int32_t* flags) {
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < ndof;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flags[g] = dof_eq[g] >= 0 ? 1 : 0;
}

__global__ void check_numbering_kernel(const int32_t* dof_eq, const int32_t* scan, int64_t ndof,
                                       int* flag) {
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < ndof;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t eq = dof_eq[g];
    if (eq >= 0 && eq != scan[g]) atomicExch(flag, 1);
    if (eq < -1) atomicExch(flag, 1);
  }
}

// Free-component mask of every element node, so the row gather needs no connectivity
// lookup before it knows which columns of a block exist.
__global__ void node_info_kernel(const int32_t* dof_eq, int64_t n_nodes, uint8_t* mask,
                                 int32_t* eq0) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int m = 0;
    int32_t first = -1;
    for (int d = 0; d < 3; ++d) {
      const int32_t eq = dof_eq[3 * a + d];
      if (eq >= 0) {
        m |= 1 << d;
        if (first < 0) first = eq;
      }
    }
    mask[a] = static_cast<uint8_t>(m);
    eq0[a] = first;
  }
}

__global__ void pair_keys_kernel(const int32_t* conn, int64_t n_elems, int npe, uint64_t N,
                                 uint64_t* keys) {
  const int64_t total = n_elems * npe * npe;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t e = i / (npe * npe);
    const int r = static_cast<int>(i % (npe * npe));
    const int a = r / npe, b = r % npe;
    keys[i] = static_cast<uint64_t>(conn[e * npe + a]) * N + static_cast<uint64_t>(conn[e * npe + b]);
  }
}

__global__ void node_ptr_kernel(const uint64_t* uniq, int64_t M, int64_t n_nodes, uint64_t N,
                                int64_t* node_ptr) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a <= n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t key = static_cast<uint64_t>(a) * N;
    int64_t lo = 0, hi = M;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (uniq[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    node_ptr[a] = lo;
  }
}

__global__ void rowlen_kernel(const uint64_t* uniq, const int64_t* node_ptr, int64_t n_nodes,
                              uint64_t N, const uint8_t* mask, int32_t* rowlen, int32_t* adj_off,
                              int64_t* node_nnz) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t run = 0;
    for (int64_t t = node_ptr[a]; t < node_ptr[a + 1]; ++t) {
      adj_off[t] = run;
      run += __popc(mask[uniq[t] % N]);
    }
    rowlen[a] = run;
    node_nnz[a] = static_cast<int64_t>(__popc(mask[a])) * run;
  }
}

__global__ void row_ptr_kernel(int64_t n_nodes, const uint8_t* mask, const int32_t* eq0,
                               const int64_t* node_base, const int32_t* rowlen, int64_t* row_ptr) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int nf = __popc(mask[a]);
    for (int r = 0; r < nf; ++r) row_ptr[eq0[a] + r] = node_base[a] + static_cast<int64_t>(r) * rowlen[a];
  }
}

__global__ void col_idx_kernel(const uint64_t* uniq, int64_t M, uint64_t N, const uint8_t* mask,
                               const int32_t* eq0, const int64_t* node_base, const int32_t* rowlen,
                               const int32_t* adj_off, int32_t* col_idx) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < M;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = static_cast<int64_t>(uniq[t] / N);
    const int64_t b = static_cast<int64_t>(uniq[t] % N);
    const int nfa = __popc(mask[a]);
    const int nfb = __popc(mask[b]);
    for (int r = 0; r < nfa; ++r) {
      const int64_t pos = node_base[a] + static_cast<int64_t>(r) * rowlen[a] + adj_off[t];
      for (int j = 0; j < nfb; ++j) col_idx[pos + j] = eq0[b] + j;
    }
  }
}

__global__ void slot_kernel(const int32_t* conn, int64_t n_elems, int npe, uint64_t N,
                            const uint64_t* uniq, const int64_t* node_ptr, uint16_t* slot, int* overflow) {
  const int64_t total = n_elems * npe * npe;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t e = i / (npe * npe);
    const int r = static_cast<int>(i % (npe * npe));
    const int64_t na = conn[e * npe + r / npe];
    const uint64_t key = static_cast<uint64_t>(na) * N + static_cast<uint64_t>(conn[e * npe + r % npe]);
    int64_t lo = node_ptr[na], hi = node_ptr[na + 1];
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (uniq[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int64_t pos = lo - node_ptr[na];
    if (pos > 65534) atomicExch(overflow, 1);  // list lengths are uint16
    slot[i] = static_cast<uint16_t>(pos);
  }
}

// adjacency list length per node (uint16, and int64 for the max reduction), and the
// list length again for the nodes whose rows are compressed (row length != 3 x list
// length), 0 for the others
__global__ void adj_len_kernel(const int64_t* node_ptr, const int32_t* rowlen, int64_t n_nodes, uint16_t* adj_len,
                               int64_t* len64, int64_t* bnd_len) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = node_ptr[a + 1] - node_ptr[a];
    adj_len[a] = static_cast<uint16_t>(k);
    len64[a] = k;
    bnd_len[a] = rowlen[a] == 3 * k ? 0 : k;
  }
}

// neighbours of the compressed-row nodes, in list order
__global__ void bnd_node_kernel(const uint64_t* uniq, int64_t M, uint64_t N, const int64_t* node_ptr,
                                const int64_t* bnd_ptr, int32_t* bnd_node) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < M;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = static_cast<int64_t>(uniq[t] / N);
    if (bnd_ptr[a + 1] > bnd_ptr[a]) bnd_node[bnd_ptr[a] + (t - node_ptr[a])] = static_cast<int32_t>(uniq[t] % N);
  }
}

__global__ void iota_kernel(int32_t* v, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[i] = static_cast<int32_t>(i);
}

__global__ void inc_ptr_kernel(const int32_t* sorted_nodes, int64_t m, int64_t n_nodes, int64_t* ptr) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a <= n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (sorted_nodes[mid] < a)
        lo = mid + 1;
      else
        hi = mid;
    }
    ptr[a] = lo;
  }
}

unsigned grid_for(int64_t n, int threads = 256) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 65536)));
}

template <typename T>
cudaError_t dalloc(T** p, size_t count, int64_t* bytes) {
  *bytes += static_cast<int64_t>(count * sizeof(T));
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

#define CXG_TRY(expr)                                  \
  do {                                                 \
    cudaError_t _e = (expr);                           \
    if (_e != cudaSuccess) {                           \
      *msg = cudaGetErrorString(_e);                   \
      rc = _e == cudaErrorMemoryAllocation ? 3 : 2;    \
      goto done;                                       \
    }                                                  \
  } while (0)

int build_pattern(int elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* d_conn,
                  const int32_t* d_dof_eq, int32_t n_free, PatternOut* out, const char** msg,
                  cudaStream_t s) {
  const int npe = nodes_of(elem_type);
  const uint64_t N = static_cast<uint64_t>(n_nodes);
  const int64_t ndof = 3 * n_nodes;
  const int64_t P = n_elems * npe * npe;
  int rc = 0;
  int64_t scratch = 0;
  int* d_flag = nullptr;
  unsigned long long* d_bad = nullptr;
  int32_t* d_flags = nullptr;
  int32_t* d_scan = nullptr;
  uint64_t* d_keys = nullptr;
  uint64_t* d_keys2 = nullptr;
  void* d_temp = nullptr;
  size_t temp_bytes = 0;
  int64_t* d_M = nullptr;
  int64_t* d_node_ptr = nullptr;
  int32_t* d_adj_off = nullptr;
  int64_t* d_node_nnz = nullptr;
  int h_flag = 0;
  int64_t M = 0;
  uint64_t* uniq = nullptr;
  unsigned long long h_bad = 0;
  int end_bit = 1;

  if (P >= (static_cast<int64_t>(1) << 31)) {
    *msg = "mesh too large for one plan (n_elems * nodes^2 >= 2^31); split it into partitions";
    return 5;
  }
  if (n_nodes >= (static_cast<int64_t>(1) << 31)) {
    *msg = "node count exceeds int32 indexing";
    return 5;
  }
  while (end_bit < 64 && (N * N) >> end_bit) ++end_bit;

  CXG_TRY(cudaMalloc(&d_flag, sizeof(int)));
  CXG_TRY(cudaMalloc(&d_bad, sizeof(unsigned long long)));
  CXG_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
  CXG_TRY(cudaMemsetAsync(d_bad, 0xff, sizeof(unsigned long long), s));

  // connectivity range check
  check_conn_kernel<<<grid_for(n_elems * npe), 256, 0, s>>>(d_conn, n_elems * npe, n_nodes, d_flag, d_bad, npe);
  CXG_TRY(cudaGetLastError());
  CXG_TRY(cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  CXG_TRY(cudaMemcpyAsync(&h_bad, d_bad, sizeof(h_bad), cudaMemcpyDeviceToHost, s));
  CXG_TRY(cudaStreamSynchronize(s));
  if (h_flag) {
    static thread_local char buf[160];
    snprintf(buf, sizeof buf, "element references unknown node (element index %llu)", h_bad);
    *msg = buf;
    rc = 6;
    goto done;
  }

  // free numbering must be ascending in g (SPC-only constraint transform)
  CXG_TRY(cudaMalloc(&d_flags, sizeof(int32_t) * std::max<int64_t>(ndof, 1)));
  CXG_TRY(cudaMalloc(&d_scan, sizeof(int32_t) * std::max<int64_t>(ndof, 1)));
  free_flags_kernel<<<grid_for(ndof), 256, 0, s>>>(d_dof_eq, ndof, d_flags);
  CXG_TRY(cudaGetLastError());
  CXG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, d_flags, d_scan, static_cast<int>(ndof), s));
  CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
  CXG_TRY(cub::DeviceScan::ExclusiveSum(d_temp, temp_bytes, d_flags, d_scan, static_cast<int>(ndof), s));
  check_numbering_kernel<<<grid_for(ndof), 256, 0, s>>>(d_dof_eq, d_scan, ndof, d_flag);
  CXG_TRY(cudaGetLastError());
  {
    int32_t last_scan = 0, last_flag = 0;
    if (ndof > 0) {
      CXG_TRY(cudaMemcpyAsync(&last_scan, d_scan + ndof - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CXG_TRY(cudaMemcpyAsync(&last_flag, d_flags + ndof - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    }
    CXG_TRY(cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CXG_TRY(cudaStreamSynchronize(s));
    if (h_flag || last_scan + last_flag != n_free) {
      *msg = "dof_eq must number the free DOFs 0..n_free-1 in increasing global DOF order "
             "(SPC-only constraint transform)";
      rc = 5;
      goto done;
    }
  }
  cudaFree(d_temp);
  d_temp = nullptr;
  cudaFree(d_flags);
  d_flags = nullptr;
  cudaFree(d_scan);
  d_scan = nullptr;

  CXG_TRY(dalloc(&out->node_mask, n_nodes, &out->device_bytes));
  CXG_TRY(dalloc(&out->node_eq0, n_nodes, &out->device_bytes));
  CXG_TRY(dalloc(&out->node_rowlen, n_nodes, &out->device_bytes));
  CXG_TRY(dalloc(&out->node_base, n_nodes, &out->device_bytes));
  node_info_kernel<<<grid_for(n_nodes), 256, 0, s>>>(d_dof_eq, n_nodes, out->node_mask, out->node_eq0);
  CXG_TRY(cudaGetLastError());

  // node adjacency by sort + unique of the element node-pair keys
  CXG_TRY(dalloc(&d_keys, P, &scratch));
  CXG_TRY(dalloc(&d_keys2, P, &scratch));
  pair_keys_kernel<<<grid_for(P), 256, 0, s>>>(d_conn, n_elems, npe, N, d_keys);
  CXG_TRY(cudaGetLastError());
  {
    cub::DoubleBuffer<uint64_t> db(d_keys, d_keys2);
    temp_bytes = 0;
    CXG_TRY(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, db, static_cast<int>(P), 0, end_bit, s));
    CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
    CXG_TRY(cub::DeviceRadixSort::SortKeys(d_temp, temp_bytes, db, static_cast<int>(P), 0, end_bit, s));
    cudaFree(d_temp);
    d_temp = nullptr;
    uint64_t* sorted = db.Current();
    uint64_t* other = db.Alternate();
    CXG_TRY(cudaMalloc(&d_M, sizeof(int64_t)));
    temp_bytes = 0;
    CXG_TRY(cub::DeviceSelect::Unique(nullptr, temp_bytes, sorted, other, d_M, static_cast<int>(P), s));
    CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
    CXG_TRY(cub::DeviceSelect::Unique(d_temp, temp_bytes, sorted, other, d_M, static_cast<int>(P), s));
    CXG_TRY(cudaMemcpyAsync(&M, d_M, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CXG_TRY(cudaStreamSynchronize(s));
    cudaFree(d_temp);
    d_temp = nullptr;
    uniq = other;
  }

  CXG_TRY(dalloc(&d_node_ptr, n_nodes + 1, &scratch));
  CXG_TRY(dalloc(&d_adj_off, M, &scratch));
  CXG_TRY(dalloc(&d_node_nnz, n_nodes, &scratch));
  node_ptr_kernel<<<grid_for(n_nodes + 1), 256, 0, s>>>(uniq, M, n_nodes, N, d_node_ptr);
  CXG_TRY(cudaGetLastError());
  rowlen_kernel<<<grid_for(n_nodes), 256, 0, s>>>(uniq, d_node_ptr, n_nodes, N, out->node_mask,
                                                  out->node_rowlen, d_adj_off, d_node_nnz);
  CXG_TRY(cudaGetLastError());
  temp_bytes = 0;
  CXG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, d_node_nnz, out->node_base, static_cast<int>(n_nodes), s));
  CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
  CXG_TRY(cub::DeviceScan::ExclusiveSum(d_temp, temp_bytes, d_node_nnz, out->node_base, static_cast<int>(n_nodes), s));
  {
    int64_t last_base = 0, last_nnz = 0;
    if (n_nodes > 0) {
      CXG_TRY(cudaMemcpyAsync(&last_base, out->node_base + n_nodes - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      CXG_TRY(cudaMemcpyAsync(&last_nnz, d_node_nnz + n_nodes - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    CXG_TRY(cudaStreamSynchronize(s));
    out->nnz = last_base + last_nnz;
  }

  CXG_TRY(dalloc(&out->row_ptr, static_cast<size_t>(n_free) + 1, &out->device_bytes));
  CXG_TRY(dalloc(&out->col_idx, static_cast<size_t>(out->nnz), &out->device_bytes));
  CXG_TRY(dalloc(&out->slot, static_cast<size_t>(P), &out->device_bytes));
  row_ptr_kernel<<<grid_for(n_nodes), 256, 0, s>>>(n_nodes, out->node_mask, out->node_eq0, out->node_base,
                                                   out->node_rowlen, out->row_ptr);
  CXG_TRY(cudaGetLastError());
  CXG_TRY(cudaMemcpyAsync(out->row_ptr + n_free, &out->nnz, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  col_idx_kernel<<<grid_for(M), 256, 0, s>>>(uniq, M, N, out->node_mask, out->node_eq0, out->node_base,
                                             out->node_rowlen, d_adj_off, out->col_idx);
  CXG_TRY(cudaGetLastError());
  CXG_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
  slot_kernel<<<grid_for(P), 256, 0, s>>>(d_conn, n_elems, npe, N, uniq, d_node_ptr, out->slot, d_flag);
  CXG_TRY(cudaGetLastError());
  CXG_TRY(cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  CXG_TRY(cudaStreamSynchronize(s));
  if (h_flag) {
    *msg = "a node has more than 65535 neighbours; not supported";
    rc = 5;
    goto done;
  }

  // largest per-node row block (free rows x row length) and adjacency list (they size
  // the gather's buffers); list lengths, and the neighbours of the compressed-row nodes
  {
    int64_t* d_max = nullptr;
    int64_t* d_bnd_len = nullptr;
    CXG_TRY(cudaMalloc(&d_max, 2 * sizeof(int64_t)));
    CXG_TRY(cudaMalloc(&d_bnd_len, sizeof(int64_t) * static_cast<size_t>(std::max<int64_t>(n_nodes, 1))));
    temp_bytes = 0;
    CXG_TRY(cub::DeviceReduce::Max(nullptr, temp_bytes, d_node_nnz, d_max, static_cast<int>(n_nodes), s));
    size_t scan_bytes = 0;
    CXG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_bnd_len, d_bnd_len, static_cast<int>(n_nodes) + 1, s));
    temp_bytes = std::max(temp_bytes, scan_bytes);
    CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
    CXG_TRY(cub::DeviceReduce::Max(d_temp, temp_bytes, d_node_nnz, d_max, static_cast<int>(n_nodes), s));
    CXG_TRY(dalloc(&out->adj_len, n_nodes, &out->device_bytes));
    CXG_TRY(dalloc(&out->bnd_ptr, n_nodes + 1, &out->device_bytes));
    adj_len_kernel<<<grid_for(n_nodes), 256, 0, s>>>(d_node_ptr, out->node_rowlen, n_nodes, out->adj_len, d_node_nnz,
                                                     d_bnd_len);
    CXG_TRY(cudaGetLastError());
    CXG_TRY(cub::DeviceReduce::Max(d_temp, temp_bytes, d_node_nnz, d_max + 1, static_cast<int>(n_nodes), s));
    CXG_TRY(cudaMemsetAsync(out->bnd_ptr + n_nodes, 0, sizeof(int64_t), s));
    CXG_TRY(cub::DeviceScan::ExclusiveSum(d_temp, temp_bytes, d_bnd_len, out->bnd_ptr, static_cast<int>(n_nodes), s));
    int64_t hm[2] = {0, 0}, last[2] = {0, 0};
    CXG_TRY(cudaMemcpyAsync(hm, d_max, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (n_nodes > 0) {
      CXG_TRY(cudaMemcpyAsync(&last[0], out->bnd_ptr + n_nodes - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      CXG_TRY(cudaMemcpyAsync(&last[1], d_bnd_len + n_nodes - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    CXG_TRY(cudaStreamSynchronize(s));
    const int64_t n_bnd = last[0] + last[1];
    CXG_TRY(cudaMemcpyAsync(out->bnd_ptr + n_nodes, &n_bnd, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    CXG_TRY(dalloc(&out->bnd_node, n_bnd, &out->device_bytes));
    bnd_node_kernel<<<grid_for(M), 256, 0, s>>>(uniq, M, N, d_node_ptr, out->bnd_ptr, out->bnd_node);
    CXG_TRY(cudaGetLastError());
    CXG_TRY(cudaStreamSynchronize(s));
    out->max_row = n_nodes > 0 ? hm[0] : 0;
    out->max_adj = n_nodes > 0 ? hm[1] : 0;
    cudaFree(d_max);
    cudaFree(d_bnd_len);
    cudaFree(d_temp);
    d_temp = nullptr;
  }

  // node -> element incidence: stable sort of (node, e*n + local) by node
  {
    const int64_t m = n_elems * npe;
    int32_t *d_codes = nullptr, *d_nodes_sorted = nullptr;
    CXG_TRY(dalloc(&out->inc_ptr, n_nodes + 1, &out->device_bytes));
    CXG_TRY(dalloc(&out->inc_code, m, &out->device_bytes));
    CXG_TRY(cudaMalloc(&d_codes, sizeof(int32_t) * std::max<int64_t>(m, 1)));
    CXG_TRY(cudaMalloc(&d_nodes_sorted, sizeof(int32_t) * std::max<int64_t>(m, 1)));
    iota_kernel<<<grid_for(m), 256, 0, s>>>(d_codes, m);
    CXG_TRY(cudaGetLastError());
    int node_bits = 1;
    while (node_bits < 31 && (n_nodes >> node_bits) != 0) ++node_bits;
    temp_bytes = 0;
    CXG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, d_conn, d_nodes_sorted, d_codes, out->inc_code,
                                            static_cast<int>(m), 0, node_bits, s));
    CXG_TRY(cudaMalloc(&d_temp, temp_bytes));
    CXG_TRY(cub::DeviceRadixSort::SortPairs(d_temp, temp_bytes, d_conn, d_nodes_sorted, d_codes, out->inc_code,
                                            static_cast<int>(m), 0, node_bits, s));
    inc_ptr_kernel<<<grid_for(n_nodes + 1), 256, 0, s>>>(d_nodes_sorted, m, n_nodes, out->inc_ptr);
    CXG_TRY(cudaGetLastError());
    CXG_TRY(cudaStreamSynchronize(s));
    cudaFree(d_codes);
    cudaFree(d_nodes_sorted);
  }

done:
  cudaFree(d_temp);
  cudaFree(d_flag);
  cudaFree(d_bad);
  cudaFree(d_flags);
  cudaFree(d_scan);
  cudaFree(d_keys);
  cudaFree(d_keys2);
  cudaFree(d_M);
  cudaFree(d_node_ptr);
  cudaFree(d_adj_off);
  cudaFree(d_node_nnz);
  return rc;
}

}  // namespace cxg
