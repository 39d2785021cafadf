// Distributed N^3 cubes over a thread-block cluster.
//
// A cluster of C CTAs holds one complex N^3 cube in shared memory, P = N/C
// planes per CTA.  Two layouts are used:
//   X-slab  (spectral side): CTA c owns lx in [cP, cP+P); local [lx-cP][ly][lz]
//   Y-slab  (real side):     CTA c owns y  in [cP, cP+P); local [y-cP][x][z]
// Rows are padded to N+1 complex elements so that one-row-per-thread access
// is bank-conflict free.  A 3-D transform is two local 1-D passes (z, y) on
// the X-slab, one exchange through distributed shared memory (each CTA stores
// its y-pencils straight into the owners' Y-slabs), and one local pass (x) on
// the Y-slab -- or the same in reverse for the forward direction.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_reg.cuh"

namespace dgfs {

template <int N, int C> struct Geo {
  static_assert(N % C == 0, "cluster size must divide N");
  static constexpr int P = N / C;         // planes per CTA
  static constexpr int ROW = N + 1;       // padded row (complex elements)
  static constexpr int PLANE = N * ROW;   // padded plane
  static constexpr int SLAB = P * PLANE;  // complex elements per slab
  static constexpr int NT = P * N;        // threads: one pencil each
  static constexpr int n = N * N * N;
};

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  cluster_arrive();
  cluster_wait();
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
template <typename T>
__device__ __forceinline__ T* peer_ptr(T* p, unsigned rank) {
  return cooperative_groups::this_cluster().map_shared_rank(p, rank);
}

// Row (z) pass on an X-slab: thread t owns row (pl = t/N, ly = t%N).
template <typename R, int N, int C, int SIGN>
__device__ __forceinline__ void slab_row_pass(c2_t<R>* A, int t) {
  using G = Geo<N, C>;
  c2_t<R> v[N];
  const int base = (t / N) * G::PLANE + (t % N) * G::ROW;
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = A[base + k];
  fft<R, N, SIGN>(v);
#pragma unroll
  for (int k = 0; k < N; ++k) A[base + k] = v[k];
}

// Column (y) pass on an X-slab: thread t owns column (pl = t/N, z = t%N);
// the transformed column is left in v.
template <typename R, int N, int C, int SIGN>
__device__ __forceinline__ void slab_col_load_fft(const c2_t<R>* A, int t,
                                                  c2_t<R>* v) {
  using G = Geo<N, C>;
  const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = A[base + k * G::ROW];
  fft<R, N, SIGN>(v);
}

// Exchange X-slab columns into the Y-slab receive buffers of their owners.
// Thread t holds v[y] for lx = rank*P + t/N, z = t%N.
template <typename R, int N, int C>
__device__ __forceinline__ void push_cols_to_yslab(c2_t<R>* Rbuf, int t,
                                                   unsigned rank,
                                                   const c2_t<R>* v) {
  using G = Geo<N, C>;
  const int lx = rank * G::P + t / N, z = t % N;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    c2_t<R>* dst = peer_ptr(Rbuf, (unsigned)c);
#pragma unroll
    for (int j = 0; j < G::P; ++j)
      dst[j * G::PLANE + lx * G::ROW + z] = v[c * G::P + j];
  }
}

// Exchange Y-slab x-pencils into the X-slab buffers of their owners.
// Thread t holds v[lx] for y = rank*P + t/N, z = t%N.
template <typename R, int N, int C>
__device__ __forceinline__ void push_pencils_to_xslab(c2_t<R>* Abuf, int t,
                                                      unsigned rank,
                                                      const c2_t<R>* v) {
  using G = Geo<N, C>;
  const int y = rank * G::P + t / N, z = t % N;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    c2_t<R>* dst = peer_ptr(Abuf, (unsigned)c);
#pragma unroll
    for (int j = 0; j < G::P; ++j)
      dst[j * G::PLANE + y * G::ROW + z] = v[c * G::P + j];
  }
}

// Load the x-pencil of thread t from a Y-slab buffer.
template <typename R, int N, int C>
__device__ __forceinline__ void yslab_load_pencil(const c2_t<R>* Rbuf, int t,
                                                  c2_t<R>* v) {
  using G = Geo<N, C>;
  const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = Rbuf[base + k * G::ROW];
}

// Slab element j (dense order within the CTA's P*N*N block) -> padded index.
template <int N, int C>
__device__ __forceinline__ int slab_index(int j) {
  using G = Geo<N, C>;
  return (j / (N * N)) * G::PLANE + ((j / N) % N) * G::ROW + (j % N);
}

}  // namespace dgfs

namespace dgfs {

// 32-bit shared-window addressing for distributed shared memory stores.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t mapa_u32(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n"
               : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};\n"
               :: "r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t addr, double2 v) {
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};\n"
               :: "r"(addr), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

}  // namespace dgfs
