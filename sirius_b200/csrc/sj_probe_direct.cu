// DISTINCT probe with a direct write-out, for the common output shapes:
//   build side: row ids plus up to 3 build payloads, either the 8-byte attached fields of the
//               table's row store (record = [row id | pad | field 0 | field 1 | field 2], one
//               load per match) or plain 4/8-byte columns without NULLs gathered by row id;
//   probe side: row ids plus up to 2 plain 4/8-byte payload columns without NULLs.
// Other shapes (NULL payloads, 1/2-byte payloads, more columns) take the staged write-out kernel
// in sj_probe.cu.
//
// Layout of the work: a warp owns 32*R consecutive probe rows and lane l handles rows
// base + 32*j + l (j < R), so every load of keys, probe payloads and partition row ids is one
// fully coalesced warp access. After probing, the warp's hits for row group j are ranked with one
// __ballot_sync: hit lanes of group j write positions off_j + popc(ballot_j & lanes below), so the
// 32 lanes of a group store one contiguous run of every output column — no shared-memory staging
// and no per-match shuffles. Output ranges are reserved with one atomicAdd per CTA tile (or per
// warp for small probes). All gather loads of a tile (records, payloads, row ids) are issued
// before the first store, so each lane keeps 3R-5R independent loads in flight.
#include <algorithm>

#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_probe_direct.h"

namespace sj {

TableDev table_dev(const sj_table* t);

constexpr int kDirectThreads = 256;
constexpr int kDirectWarps = kDirectThreads / 32;

__device__ __forceinline__ uint64_t ld_cs_w(const void* base, int64_t i, int w) {
  return w == 8 ? __ldcs(reinterpret_cast<const unsigned long long*>(base) + i)
                : (uint64_t)__ldcs(reinterpret_cast<const unsigned int*>(base) + i);
}
__device__ __forceinline__ uint64_t ld_nc_w(const void* a, int w) {
  return w == 8 ? __ldg(reinterpret_cast<const unsigned long long*>(a))
                : (uint64_t)__ldg(reinterpret_cast<const unsigned int*>(a));
}
__device__ __forceinline__ void st_cs_w(void* base, int64_t i, int w, uint64_t v) {
  if (w == 8) __stcs(reinterpret_cast<unsigned long long*>(base) + i, (unsigned long long)v);
  else __stcs(reinterpret_cast<unsigned int*>(base) + i, (unsigned int)v);
}

// One row-store record of 8, 16 or 32 bytes (the stride) in one load.
__device__ __forceinline__ void load_rec(const void* p, int stride, uint32_t (&w)[8]) {
  if (stride == 32) {
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p));
  } else if (stride == 16) {
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
    w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
    w[4] = w[5] = w[6] = w[7] = 0;
  } else {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
    w[0] = x.x; w[1] = x.y;
    w[2] = w[3] = w[4] = w[5] = w[6] = w[7] = 0;
  }
}

template <typename K, bool WIDE, int R, bool CTA_AGG>
__global__ void __launch_bounds__(kDirectThreads, (R <= 2 ? 4 : 2))
    probe_direct_kernel(TableDev t, const K* __restrict__ keys, const uint32_t* __restrict__ kv, int64_t kvoff,
                        int64_t n_host, const int64_t* d_n, DirectArgs a) {
  using Ops = SlotOps<WIDE>;
  __shared__ unsigned s_wtot[kDirectWarps];
  __shared__ unsigned long long s_wbase[kDirectWarps];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  const int64_t n = d_n ? *d_n : n_host;
  constexpr int64_t kRowsCta = (int64_t)kDirectThreads * R;
  const int64_t tiles = (n + kRowsCta - 1) / kRowsCta;
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t r0 = tile * kRowsCta + (int64_t)warp * (32 * R) + lane;  // row of group j: r0 + 32 j
    K k[R];
#pragma unroll
    for (int j = 0; j < R; ++j) k[j] = r0 + 32 * j < n ? __ldcs(keys + r0 + 32 * j) : (K)0;
    uint32_t act = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t r = r0 + 32 * j;
      if (r < n && bit_valid(kv, kvoff, r) && in_range(t, k[j])) act |= 1u << j;
    }
    uint32_t b[R];
    uint64_t ks[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint64_t kb = key_u64<K>(k[j]);
      b[j] = home_bucket(t, kb);
      ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
    }
    int32_t pos[R];
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) pos[j] = 0;
    for (uint32_t step = 0; act && step <= t.segmask; ++step) {
      Bucket bk[R];
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (act >> j & 1u) bk[j] = load_bucket<true>(t.slots, b[j]);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (!(act >> j & 1u)) continue;
        bool done = false;
#pragma unroll
        for (int q = 0; q < Ops::kSlots; ++q) {
          if (!done && Ops::match_s(bk[j], q, ks[j], kmask)) {
            pos[j] = Ops::rid(bk[j], q, t.rbits);
            hit |= 1u << j;
            done = true;
          }
          done |= Ops::empty(bk[j], q);
        }
        if (done) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    unsigned bal[R];
    unsigned wtot = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      bal[j] = __ballot_sync(kFullMask, (hit >> j) & 1u);
      wtot += __popc(bal[j]);
    }
    unsigned long long base;
    if (CTA_AGG) {
      if (lane == 0) s_wtot[warp] = wtot;
      __syncthreads();
      if (warp == 0) {
        const unsigned v = lane < kDirectWarps ? s_wtot[lane] : 0u;
        unsigned incl = v;
#pragma unroll
        for (int d = 1; d < kDirectWarps; d <<= 1) {
          const unsigned o = __shfl_up_sync(kFullMask, incl, d);
          if (lane >= d) incl += o;
        }
        const unsigned tot = __shfl_sync(kFullMask, incl, kDirectWarps - 1);
        unsigned long long cb = 0;
        if (lane == 0 && tot) cb = atomicAdd(a.d_count, (unsigned long long)tot);
        cb = __shfl_sync(kFullMask, cb, 0);
        if (lane < kDirectWarps) s_wbase[lane] = cb + (incl - v);
      }
      __syncthreads();
      base = s_wbase[warp];
    } else {
      base = 0;
      if (lane == 0 && wtot) base = atomicAdd(a.d_count, (unsigned long long)wtot);
      base = __shfl_sync(kFullMask, base, 0);
    }
    if (wtot == 0) continue;

    // ---- gather loads for every hit of the tile ----
    int64_t p[R];
    {
      unsigned run = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        p[j] = (int64_t)(base + run + __popc(bal[j] & below));
        run += __popc(bal[j]);
      }
    }
    int32_t prid[R], brid[R];
    uint64_t pv[kDirectMaxProbePayload][R];
    uint64_t bv[kDirectMaxBuildPayload][R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      prid[j] = brid[j] = 0;
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c) pv[c][j] = 0;
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c) bv[c][j] = 0;
      if (!(hit >> j & 1u)) continue;
      const int64_t r = r0 + 32 * j;
      if (a.out_prid) prid[j] = a.prid_map ? __ldcs(a.prid_map + r) : (int32_t)r;
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c)
        if (c < a.n_pin) pv[c][j] = ld_cs_w(a.pin[c], r, a.pin_w[c]);
      if (a.rec) {
        uint32_t w[8];
        load_rec(static_cast<const char*>(a.rec) + (int64_t)pos[j] * a.rec_stride, a.rec_stride, w);
        brid[j] = (int32_t)w[0];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c)
          bv[c][j] = ((uint64_t)w[3 + 2 * c] << 32) | w[2 + 2 * c];
      } else {
        brid[j] = a.brid_map ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(a.brid_map) +
                                                                       (int64_t)pos[j] * a.brid_stride))
                             : pos[j];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c) {
          if (c < a.n_bin) {
            const int64_t i = a.bin_by_pos ? pos[j] : brid[j];
            bv[c][j] = ld_nc_w(static_cast<const char*>(a.bin[c]) + i * a.bin_stride[c], a.bin_w[c]);
          }
        }
      }
    }
    // ---- stores: each row group j is one contiguous run of positions per column ----
#pragma unroll
    for (int j = 0; j < R; ++j) {
      if (!(hit >> j & 1u) || p[j] >= a.capacity) continue;
      if (a.out_prid) __stcs(a.out_prid + p[j], prid[j]);
      if (a.out_brid) __stcs(a.out_brid + p[j], brid[j]);
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c)
        if (c < a.n_pin) st_cs_w(a.pout[c], p[j], a.pin_w[c], pv[c][j]);
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c)
        if (c < a.n_bin) st_cs_w(a.bout[c], p[j], a.bin_w[c], bv[c][j]);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
bool direct_args(const GatherArgs& g, DirectArgs& a) {
  if (g.n_pin > kDirectMaxProbePayload || g.n_bin > kDirectMaxBuildPayload) return false;
  a = DirectArgs{};
  a.out_prid = g.out_prid;
  a.out_brid = g.out_brid;
  a.prid_map = g.prid_map;
  a.capacity = g.capacity;
  a.d_count = g.d_count;
  a.n_pin = g.n_pin;
  a.n_bin = g.n_bin;
  for (int c = 0; c < g.n_pin; ++c) {
    const PayloadIn& in = g.pin[c];
    if (in.valid || in.valid8 || (in.width != 4 && in.width != 8) || in.stride != in.width) return false;
    a.pin[c] = in.data;
    a.pin_w[c] = in.width;
    a.pout[c] = g.pout[c].data;
  }
  if (g.n_bin > 0 && g.rec) {
    if (g.rec_stride != 16 && g.rec_stride != 32) return false;
    for (int c = 0; c < g.n_bin; ++c)
      if (g.bin[c].width != 8 || g.rec_voff[c] >= 0 || g.rec_off[c] != 8 + 8 * c) return false;
    a.rec = g.rec;
    a.rec_stride = g.rec_stride;
    for (int c = 0; c < g.n_bin; ++c) {
      a.bin_w[c] = 8;
      a.bout[c] = g.bout[c].data;
    }
    return true;
  }
  a.brid_map = g.brid_map;
  a.brid_stride = g.brid_stride;
  a.bin_by_pos = g.bin_by_pos;
  for (int c = 0; c < g.n_bin; ++c) {
    const PayloadIn& in = g.bin[c];
    if (in.valid || in.valid8 || (in.width != 4 && in.width != 8)) return false;
    a.bin[c] = in.data;
    a.bin_stride[c] = in.stride;
    a.bin_w[c] = in.width;
    a.bout[c] = g.bout[c].data;
  }
  return true;
}

template <typename K, bool WIDE, int R, bool CTA>
static void launch_direct_kernel(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a,
                                 cudaStream_t s) {
  static int resident = 0;  // CTAs per SM of this instantiation (same on every B200)
  if (resident == 0) {
    int r = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, probe_direct_kernel<K, WIDE, R, CTA>, kDirectThreads, 0);
    resident = std::max(1, r);
  }
  const int64_t tiles = (p.num_rows + (int64_t)kDirectThreads * R - 1) / ((int64_t)kDirectThreads * R);
  const int per_sm = std::min(resident, std::max(1, t->params.ctas_per_sm));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count(t->device) * per_sm));
  probe_direct_kernel<K, WIDE, R, CTA><<<grid, kDirectThreads, 0, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, d_n, a);
}

template <typename K, bool WIDE>
static void launch_direct(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a, int rpl,
                          bool cta, cudaStream_t s) {
  if (rpl >= 4) {
    if (cta) launch_direct_kernel<K, WIDE, 4, true>(t, p, d_n, a, s);
    else launch_direct_kernel<K, WIDE, 4, false>(t, p, d_n, a, s);
  } else {
    if (cta) launch_direct_kernel<K, WIDE, 2, true>(t, p, d_n, a, s);
    else launch_direct_kernel<K, WIDE, 2, false>(t, p, d_n, a, s);
  }
}

bool probe_direct(const sj_table* t, const sj_column& p, const int64_t* d_n, const GatherArgs& g, cudaStream_t s) {
  const sj_join_params& pr = t->params;
  if (pr.probe_kernel == SJ_PROBE_KERNEL_STAGED) return false;
  DirectArgs a;
  if (!direct_args(g, a)) return false;
  const int agg = pr.aggregation;
  const bool cta = agg == SJ_AGG_CTA || (agg == SJ_AGG_AUTO && p.num_rows >= (1 << 20));
  const int rpl = pr.rows_per_lane > 0 ? pr.rows_per_lane : 2;
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  KernelTimer timer("probe_direct", s);
  if (t->key_type == SJ_INT32) {
    if (wide) launch_direct<int32_t, true>(t, p, d_n, a, rpl, cta, s);
    else launch_direct<int32_t, false>(t, p, d_n, a, rpl, cta, s);
  } else {
    if (wide) launch_direct<int64_t, true>(t, p, d_n, a, rpl, cta, s);
    else launch_direct<int64_t, false>(t, p, d_n, a, rpl, cta, s);
  }
  return true;
}

}  // namespace sj
