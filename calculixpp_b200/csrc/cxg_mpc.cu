// Multi-point constraints: the reduced free system of a model with slave DOFs.
//
// The reference scatters every element block through the constraint transform,
// K_ff[eqA][eqB] += cA * kab * cB over the expansion terms of both DOFs, and moves the
// expansions' constants into the rhs (src/fem/assembly.cpp:76-101; the transform is
// src/fem/constraint_transform.cpp:25-131). Here the element pass and the row gather
// assemble K_x on an extended numbering in which slave DOFs are equations as well (so the
// pattern builder, slot maps and kernels are the ordinary ones), and this file reduces it:
//   K_ff = T^T K_x T,  rhs = T^T (rhs_x - K_x c),
// with T the expansion (a free equation maps to itself with weight 1, a slave to its
// terms) and c the slaves' constants on the extended numbering. Every reduced entry is
// a fixed-order sum over a precomputed list of (extended entry, weight) pairs, so the
// result is deterministic. The pattern of K_ff is the union of the targets of every
// extended entry, built once per plan with CUB sorts.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "cxg_internal.cuh"

namespace cxg {
namespace {

unsigned grid_n(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

// Expansion of extended equation x: ext_map[x] >= 0 is a free equation (weight 1), else
// slave s = -1 - ext_map[x] with terms [term_ptr[s], term_ptr[s+1]).
struct Expansion {
  const int32_t* ext_map;
  const int64_t* term_ptr;
  const int32_t* term_eq;
  const double* term_coeff;
  __device__ int64_t count(int64_t x) const {
    const int32_t m = ext_map[x];
    if (m >= 0) return 1;
    const int32_t s = -1 - m;
    return term_ptr[s + 1] - term_ptr[s];
  }
  __device__ void term(int64_t x, int64_t i, int32_t& eq, double& c) const {
    const int32_t m = ext_map[x];
    if (m >= 0) {
      eq = m;
      c = 1.0;
      return;
    }
    const int64_t k = term_ptr[-1 - m] + i;
    eq = term_eq[k];
    c = term_coeff[k];
  }
};

__global__ void entry_rows_kernel(const int64_t* row_ptr, int64_t n_rows, int64_t* row_of) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n_rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) row_of[k] = r;
}

__global__ void count_targets_kernel(Expansion T, const int64_t* row_of, const int32_t* col, int64_t nnz,
                                     int64_t* count) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x)
    count[k] = T.count(row_of[k]) * T.count(col[k]);
}

// Every target (eqA, eqB) of extended entry k: key eqA * n_free + eqB, source k, weight cA cB.
__global__ void emit_targets_kernel(Expansion T, const int64_t* row_of, const int32_t* col, int64_t nnz,
                                    const int64_t* offset, int64_t n_free, uint64_t* key, int64_t* order,
                                    int64_t* src, double* w) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t x = row_of[k], y = col[k];
    const int64_t nx = T.count(x), ny = T.count(y);
    int64_t o = offset[k];
    for (int64_t i = 0; i < nx; ++i) {
      int32_t ea;
      double ca;
      T.term(x, i, ea, ca);
      for (int64_t j = 0; j < ny; ++j) {
        int32_t eb;
        double cb;
        T.term(y, j, eb, cb);
        key[o] = static_cast<uint64_t>(ea) * static_cast<uint64_t>(n_free) + static_cast<uint64_t>(eb);
        order[o] = o;
        src[o] = k;
        w[o] = ca * cb;
        ++o;
      }
    }
  }
}

// rhs targets of extended row x: (eq, x, c) for every term of x's expansion.
__global__ void emit_rhs_kernel(Expansion T, int64_t n_x, const int64_t* offset, uint64_t* key, int64_t* order,
                                int64_t* src, double* w) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n_x;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t o = offset[x];
    for (int64_t i = 0, n = T.count(x); i < n; ++i, ++o) {
      int32_t e;
      double c;
      T.term(x, i, e, c);
      key[o] = static_cast<uint64_t>(e);
      order[o] = o;
      src[o] = x;
      w[o] = c;
    }
  }
}

__global__ void count_x_kernel(Expansion T, int64_t n_x, int64_t* count) {
  for (int64_t x = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; x < n_x;
       x += static_cast<int64_t>(gridDim.x) * blockDim.x)
    count[x] = T.count(x);
}

__global__ void permute_kernel(const int64_t* perm, const int64_t* src_in, const double* w_in, int64_t n,
                               int64_t* src_out, double* w_out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    src_out[i] = src_in[perm[i]];
    w_out[i] = w_in[perm[i]];
  }
}

// row_ptr[r] = first unique key with key / n_free >= r (keys ascending)
__global__ void rows_from_keys_kernel(const uint64_t* ukey, int64_t n_u, int64_t n_rows, uint64_t n_free,
                                      int64_t* row_ptr, int32_t* col) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r <= n_rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t lo = static_cast<uint64_t>(r) * n_free;
    int64_t a = 0, b = n_u;
    while (a < b) {
      const int64_t m = (a + b) / 2;
      if (ukey[m] < lo) a = m + 1; else b = m;
    }
    row_ptr[r] = a;
  }
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n_u;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    col[i] = static_cast<int32_t>(ukey[i] % n_free);
}

// dense rhs pointer: ptr[e] = first list entry of equation e (keys ascending)
__global__ void ptr_from_keys_kernel(const uint64_t* key, int64_t n, int64_t n_eq, int64_t* ptr) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e <= n_eq;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t a = 0, b = n;
    while (a < b) {
      const int64_t m = (a + b) / 2;
      if (key[m] < static_cast<uint64_t>(e)) a = m + 1; else b = m;
    }
    ptr[e] = a;
  }
}

__global__ void reduce_kernel(const int64_t* ptr, const int64_t* src, const double* w, const double* x, int64_t n,
                              double* out) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int64_t k = ptr[t]; k < ptr[t + 1]; ++k) v += w[k] * x[src[k]];
    out[t] = v;
  }
}

__global__ void sub_kernel(const double* a, const double* b, int64_t n, double* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = a[i] - b[i];
}

// Sort (key, order) pairs, then gather src / w into key order: a stable sort keeps the
// emission order among equal keys, so every list is summed in a fixed order.
cudaError_t sort_lists(uint64_t* key, int64_t* order, int64_t* src, double* w, int64_t n, int end_bit,
                       uint64_t** key_sorted, int64_t** src_sorted, double** w_sorted, cudaStream_t s) {
  uint64_t* k2 = nullptr;
  int64_t* o2 = nullptr;
  void* temp = nullptr;
  size_t tb = 0;
  cudaError_t e = cudaMalloc(&k2, sizeof(uint64_t) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(&o2, sizeof(int64_t) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(src_sorted, sizeof(int64_t) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(w_sorted, sizeof(double) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb, key, k2, order, o2, n, 0, end_bit, s);
  if (e == cudaSuccess) e = cudaMalloc(&temp, std::max<size_t>(tb, 16));
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, tb, key, k2, order, o2, n, 0, end_bit, s);
  if (e == cudaSuccess) {
    permute_kernel<<<grid_n(n), 256, 0, s>>>(o2, src, w, n, *src_sorted, *w_sorted);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(o2);
  cudaFree(temp);
  *key_sorted = k2;
  return e;
}

int end_bit_for(uint64_t max_key) {
  int b = 1;
  while (b < 64 && (max_key >> b) != 0) ++b;
  return b;
}

}  // namespace

cudaError_t build_mpc_reduce(const int64_t* x_row_ptr, const int32_t* x_col, int64_t n_x, int64_t nnz_x,
                             const int32_t* ext_map, const int64_t* term_ptr, const int32_t* term_eq,
                             const double* term_coeff, int32_t n_free, MpcLists* out, cudaStream_t s) {
  Expansion T{ext_map, term_ptr, term_eq, term_coeff};
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) {
    const cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) tmp.push_back(*p);
    return e;
  };
  int64_t *row_of = nullptr, *count = nullptr, *offset = nullptr, *order = nullptr, *src = nullptr;
  uint64_t* key = nullptr;
  double* w = nullptr;
  void* temp = nullptr;
  size_t tb = 0;
  int64_t total = 0;
  cudaError_t e = alloc(reinterpret_cast<void**>(&row_of), 8 * nnz_x);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&count), 8 * (nnz_x + 1));
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&offset), 8 * (nnz_x + 1));
  if (e == cudaSuccess) {
    entry_rows_kernel<<<grid_n(n_x), 256, 0, s>>>(x_row_ptr, n_x, row_of);
    count_targets_kernel<<<grid_n(nnz_x), 256, 0, s>>>(T, row_of, x_col, nnz_x, count);
    e = cudaMemsetAsync(count + nnz_x, 0, 8, s);
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, count, offset, nnz_x + 1, s);
  if (e == cudaSuccess) e = alloc(&temp, tb);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(temp, tb, count, offset, nnz_x + 1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, offset + nnz_x, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&key), 8 * total);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&order), 8 * total);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&src), 8 * total);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&w), 8 * total);
  if (e == cudaSuccess) {
    emit_targets_kernel<<<grid_n(nnz_x), 256, 0, s>>>(T, row_of, x_col, nnz_x, offset, n_free, key, order, src, w);
    e = cudaGetLastError();
  }
  uint64_t* ks = nullptr;
  const uint64_t nf = static_cast<uint64_t>(std::max(n_free, 1));
  if (e == cudaSuccess)
    e = sort_lists(key, order, src, w, total, end_bit_for(nf * nf), &ks, &out->src, &out->w, s);
  if (ks) tmp.push_back(ks);
  // unique keys -> reduced pattern; run starts -> per-entry source lists
  uint64_t* ukey = nullptr;
  int64_t *runs = nullptr, *n_u = nullptr;
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&ukey), 8 * total);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&runs), 8 * (total + 1));
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&n_u), 8);
  size_t tb2 = 0;
  if (e == cudaSuccess) e = cub::DeviceRunLengthEncode::Encode(nullptr, tb2, ks, ukey, runs, n_u, total, s);
  void* temp2 = nullptr;
  if (e == cudaSuccess) e = alloc(&temp2, tb2);
  if (e == cudaSuccess) e = cub::DeviceRunLengthEncode::Encode(temp2, tb2, ks, ukey, runs, n_u, total, s);
  int64_t nu = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nu, n_u, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMalloc(&out->tgt_ptr, 8 * (nu + 1));
  if (e == cudaSuccess) e = cudaMemsetAsync(runs + nu, 0, 8, s);
  size_t tb3 = 0;
  void* temp3 = nullptr;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb3, runs, out->tgt_ptr, nu + 1, s);
  if (e == cudaSuccess) e = alloc(&temp3, tb3);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(temp3, tb3, runs, out->tgt_ptr, nu + 1, s);
  if (e == cudaSuccess) e = cudaMalloc(&out->row_ptr, 8 * (static_cast<size_t>(n_free) + 1));
  if (e == cudaSuccess) e = cudaMalloc(&out->col_idx, 4 * std::max<int64_t>(nu, 1));
  if (e == cudaSuccess) {
    rows_from_keys_kernel<<<grid_n(std::max<int64_t>(nu, n_free + 1)), 256, 0, s>>>(ukey, nu, n_free, nf, out->row_ptr,
                                                                                    out->col_idx);
    e = cudaGetLastError();
  }
  out->nnz = nu;
  // rhs lists: T^T over extended rows
  int64_t *xcount = nullptr, *xoff = nullptr, xtotal = 0;
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&xcount), 8 * (n_x + 1));
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&xoff), 8 * (n_x + 1));
  if (e == cudaSuccess) {
    count_x_kernel<<<grid_n(n_x), 256, 0, s>>>(T, n_x, xcount);
    e = cudaMemsetAsync(xcount + n_x, 0, 8, s);
  }
  size_t tb4 = 0;
  void* temp4 = nullptr;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb4, xcount, xoff, n_x + 1, s);
  if (e == cudaSuccess) e = alloc(&temp4, tb4);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(temp4, tb4, xcount, xoff, n_x + 1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&xtotal, xoff + n_x, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  uint64_t *rkey = nullptr, *rks = nullptr;
  int64_t *rorder = nullptr, *rsrc = nullptr;
  double* rw = nullptr;
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&rkey), 8 * xtotal);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&rorder), 8 * xtotal);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&rsrc), 8 * xtotal);
  if (e == cudaSuccess) e = alloc(reinterpret_cast<void**>(&rw), 8 * xtotal);
  if (e == cudaSuccess) {
    emit_rhs_kernel<<<grid_n(n_x), 256, 0, s>>>(T, n_x, xoff, rkey, rorder, rsrc, rw);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = sort_lists(rkey, rorder, rsrc, rw, xtotal, end_bit_for(nf), &rks, &out->rhs_src, &out->rhs_w, s);
  if (rks) tmp.push_back(rks);
  if (e == cudaSuccess) e = cudaMalloc(&out->rhs_ptr, 8 * (static_cast<size_t>(n_free) + 1));
  if (e == cudaSuccess) {
    ptr_from_keys_kernel<<<grid_n(n_free + 1), 256, 0, s>>>(rks, xtotal, n_free, out->rhs_ptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  for (void* p : tmp) cudaFree(p);
  return e;
}

cudaError_t mpc_reduce_values(const MpcLists& m, const double* vals_x, double* vals, cudaStream_t s) {
  if (m.nnz == 0) return cudaSuccess;
  reduce_kernel<<<grid_n(m.nnz), 256, 0, s>>>(m.tgt_ptr, m.src, m.w, vals_x, m.nnz, vals);
  return cudaGetLastError();
}

cudaError_t mpc_reduce_rhs(const MpcLists& m, const double* rhs_x, const double* kc, int64_t n_x, double* tmp_x,
                           int32_t n_free, double* rhs, cudaStream_t s) {
  const double* r = rhs_x;
  if (kc) {
    sub_kernel<<<grid_n(n_x), 256, 0, s>>>(rhs_x, kc, n_x, tmp_x);
    r = tmp_x;
  }
  if (n_free > 0) reduce_kernel<<<grid_n(n_free), 256, 0, s>>>(m.rhs_ptr, m.rhs_src, m.rhs_w, r, n_free, rhs);
  return cudaGetLastError();
}

}  // namespace cxg
