// net_conv_tc.cu — 3x3 convolutions of the guess network on the fifth-generation
// tensor cores (tcgen05.mma, accumulator in tensor memory, operands staged by TMA).
//
// Implicit GEMM per tile of 128 output pixels of one image row (images whose
// width is a multiple of 128):
//   D[p][co] = Σ_tap Σ_ci A_tap[p][ci] · W[tap][co][ci],  M = 128, N = COUT, K = 9·CIN
// The input halo of a tile (3 rows x 130 pixels x CIN channels, zero outside the
// image) is loaded by TMA, one box per group of 8 channels, into shared memory
// as [channel group][row][pixel][8 channels] — which is the tensor cores'
// K-major, non-swizzled operand layout (16-byte rows, 8-row core matrices 128 B
// apart, channel groups one plane apart).  The operand of tap (dy, dx) is the
// same buffer viewed from pixel (dy·130 + dx): a descriptor start 16·(dy·130 + dx)
// bytes further on, so the nine taps need no copies.  Weights [tap][co][ci] sit
// in shared memory as [tap][channel group][co][8 channels] for the whole launch.
//
// A CTA of 128 threads is persistent over tiles, with two halo buffers and two
// accumulators (64 tensor-memory columns).  Thread 0 issues the 9·CIN/16 MMAs
// of a tile (one instruction each, M = 128, N = COUT, K = 16) and commits them
// to that accumulator's mbarrier; the MMAs of tile j + 1 are issued before the
// block's epilogue of tile j, so the tensor core works while the four warps
// read accumulator j & 1 (warp w: TMEM lanes 32w..32w+31, one pixel per
// thread, COUT fp32 columns), apply bias and ReLU or the ReLU mask and store
// bf16 (or fp32) NHWC rows; the TMA of tile j + 2 goes out as soon as tile j's
// MMAs have released its halo buffer.  Every wait on an mbarrier
// is bounded; a wait that runs out sets the error word the host checks, and the
// CTA waits (bounded) for its own copies and MMAs before it frees its tensor
// memory.
//
// Weight gradients stay on the mma.sync kernel (net_kernels.cu): their GEMM has
// M = CIN = 16..32 rows per tap, below the tcgen05 minimum of 64, and the nine
// taps are shifted views that one descriptor stride cannot stack.
#include <cuda.h>

#include <mutex>

#include "net_kernels.cuh"

namespace cdm {
namespace net {

namespace {

constexpr int TP = 128;        // output pixels per tile (one image row segment)
constexpr int HP = TP + 2;     // halo pixels per row
constexpr int HROWS = 3;       // halo rows
constexpr int PLANE = 6272;    // bytes of one channel group's halo (3·130·16 = 6240, padded to 128)
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ int g_tc_error;  // set when a bounded wait runs out (read and cleared by the host)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// true once the barrier's phase with the given parity has completed; false when
// the wait ran out (about 2 s)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = now_ns();
  for (int n = 0; n < (1 << 26); ++n) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((n & 255) == 255 && now_ns() - t0 > kWaitNs) break;
  }
  return false;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// shared-memory operand descriptor: K-major, no swizzle (start, leading = next K
// core matrix, stride = next 8 rows), Blackwell descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: bf16 A and B (K-major), fp32 D, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TP >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_tc(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 (or 32) consecutive fp32 columns of this thread's TMEM lane
template <int NCOL>
__device__ __forceinline__ void tmem_load(uint32_t taddr, float* v);

template <>
__device__ __forceinline__ void tmem_load<16>(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

template <>
__device__ __forceinline__ void tmem_load<32>(uint32_t taddr, float* v) {
  tmem_load<16>(taddr, v);
  tmem_load<16>(taddr + 16, v + 16);
}

template <int CIN, int COUT>
struct TcSmem {
  static constexpr int CG = CIN / 8;
  alignas(1024) unsigned char halo[2][CG * PLANE];
  alignas(128) unsigned char w[9 * CG * COUT * 16];
  float bias[COUT];
  unsigned long long bar_tma[2];
  unsigned long long bar_mma[2];
  uint32_t tmem_base;
  int err;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap xmap, ConvArgs a,
                                                         int ntiles) {
  constexpr int CG = CIN / 8, KSTEPS = CIN / 16;
  using Smem = TcSmem<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // the struct starts on a 1024-byte boundary of the shared window (the launch adds the slack)
  const uint32_t pad = (1024u - (smem_addr(smem_raw) & 1023u)) & 1023u;
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw + pad);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_x = a.W / TP;

  // weights into [tap][channel group][co][8 channels], bias
  for (int v = tid; v < 9 * COUT * CG; v += 128) {
    const int g = v % CG, row = v / CG;  // row = tap·COUT + co
    const int tap = row / COUT, co = row - tap * COUT;
    *reinterpret_cast<uint4*>(sm.w + ((tap * CG + g) * COUT + co) * 16) =
        *reinterpret_cast<const uint4*>(a.w + (size_t)row * CIN + g * 8);
  }
  if (tid < COUT) sm.bias[tid] = a.bias ? a.bias[tid] : 0.f;
  if (tid == 0) {
    mbar_init(smem_addr(&sm.bar_tma[0]), 1);
    mbar_init(smem_addr(&sm.bar_tma[1]), 1);
    mbar_init(smem_addr(&sm.bar_mma[0]), 1);
    mbar_init(smem_addr(&sm.bar_mma[1]), 1);
    sm.err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // 64 columns of tensor memory: two fp32 accumulators (N <= 32 each)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_addr(&sm.tmem_base)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // the generic-proxy weight stores become visible to the tensor cores' reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;
  const uint32_t idesc = idesc_bf16(COUT);

  auto issue_tma = [&](int t, int buf) {
    const int b = t / (a.H * tiles_x), r = t - b * a.H * tiles_x;
    const int y = r / tiles_x, x0 = (r - y * tiles_x) * TP;
    const uint32_t bar = smem_addr(&sm.bar_tma[buf]);
    mbar_expect_tx(bar, CG * HROWS * HP * 16);
#pragma unroll
    for (int g = 0; g < CG; ++g)
      tma_load_4d(smem_addr(sm.halo[buf] + g * PLANE), &xmap, bar, 8 * g, x0 - 1, y - 1, b);
  };

  // this CTA's tiles: blockIdx.x + j·gridDim.x, j < nt
  const int nt = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile_of = [&](int j) { return (int)blockIdx.x + j * (int)gridDim.x; };
  // the nine taps' MMAs of halo buffer hb into accumulator ab, committed to bar_mma[ab]
  auto issue_mmas = [&](int hb, int ab) {
    tc_fence_after();
    const uint32_t hs = smem_addr(sm.halo[hb]), wb = smem_addr(sm.w);
    int k = 0;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dy = tap / 3, dx = tap - 3 * (tap / 3);
#pragma unroll
      for (int ks = 0; ks < KSTEPS; ++ks, ++k) {
        const uint64_t ad = smem_desc(hs + 2 * ks * PLANE + (dy * HP + dx) * 16, PLANE, 128);
        const uint64_t bd = smem_desc(wb + ((tap * CG + 2 * ks) * COUT) * 16, COUT * 16, 128);
        mma_bf16_tc(tmem + 32u * (uint32_t)ab, ad, bd, idesc, k > 0 ? 1u : 0u);
      }
    }
    mma_commit(smem_addr(&sm.bar_mma[ab]));
  };
  // Pipeline (tile j uses halo buffer and accumulator j & 1): thread 0 issues the
  // MMAs of tile j + 1 before the block's epilogue of tile j, and the TMA of tile
  // j + 2 once tile j's MMAs have released its halo buffer.  Thread 0 counts what
  // it issued and what it saw complete on each barrier, for the drain after a
  // failed wait.
  // (kept in scalars: counts indexed by buffer would live in local memory)
  int tma_n0 = 0, tma_n1 = 0, tma_w0 = 0, tma_w1 = 0, mma_n0 = 0, mma_n1 = 0, mma_w0 = 0, mma_w1 = 0;
  auto bump = [](int& c0, int& c1, int b) {
    if (b) ++c1;
    else ++c0;
  };
  bool fail = false;
  if (tid == 0) {
    for (int j = 0; j < 2 && j < nt; ++j) {
      issue_tma(tile_of(j), j);
      bump(tma_n0, tma_n1, j);
    }
    if (nt > 0) {
      if (mbar_wait(smem_addr(&sm.bar_tma[0]), 0)) {
        ++tma_w0;
        issue_mmas(0, 0);
        ++mma_n0;
      } else {
        fail = true;
      }
    }
  }
  bool failed = __syncthreads_or(fail ? 1 : 0) != 0;
  for (int j = 0; j < nt && !failed; ++j) {
    const int b = j & 1;
    if (tid == 0 && j + 1 < nt) {
      if (mbar_wait(smem_addr(&sm.bar_tma[b ^ 1]), ((j + 1) >> 1) & 1)) {
        bump(tma_w0, tma_w1, b ^ 1);
        issue_mmas(b ^ 1, b ^ 1);
        bump(mma_n0, mma_n1, b ^ 1);
      } else {
        fail = true;
      }
    }
    // this tile's MMAs (which also frees its halo buffer for tile j + 2)
    const bool ok = mbar_wait(smem_addr(&sm.bar_mma[b]), (j >> 1) & 1);
    if (tid == 0 && ok) {
      bump(mma_w0, mma_w1, b);
      if (!fail && j + 2 < nt) {
        issue_tma(tile_of(j + 2), b);
        bump(tma_n0, tma_n1, b);
      }
    }
    tc_fence_after();
    if (ok) {
      // epilogue: thread = pixel (lane 32·warp + lane of the accumulator)
      const int t = tile_of(j);
      float v[COUT];
      tmem_load<COUT>(tmem + ((uint32_t)(32 * warp) << 16) + 32u * (uint32_t)b, v);
      const int bi = t / (a.H * tiles_x), r = t - bi * a.H * tiles_x;
      const int y = r / tiles_x, x = (r - y * tiles_x) * TP + 32 * warp + lane;
      const size_t pix = ((size_t)bi * a.H + y) * a.W + x;
#pragma unroll
      for (int co = 0; co < COUT; ++co) v[co] += sm.bias[co];
      if (a.epi == EPI_RELU) {
#pragma unroll
        for (int co = 0; co < COUT; ++co) v[co] = fmaxf(v[co], 0.f);
      } else if (a.epi == EPI_MASK) {
#pragma unroll
        for (int c8 = 0; c8 < COUT / 8; ++c8) {
          const uint4 mk = *reinterpret_cast<const uint4*>(a.mask + pix * COUT + 8 * c8);
          const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(&mk);
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            if (!(__bfloat162float(m2[h].x) > 0.f)) v[8 * c8 + 2 * h] = 0.f;
            if (!(__bfloat162float(m2[h].y) > 0.f)) v[8 * c8 + 2 * h + 1] = 0.f;
          }
        }
      }
      if (a.out) {
#pragma unroll
        for (int c8 = 0; c8 < COUT / 8; ++c8) {
          uint4 o;
          __nv_bfloat162* o2 = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
          for (int h = 0; h < 4; ++h) o2[h] = __floats2bfloat162_rn(v[8 * c8 + 2 * h], v[8 * c8 + 2 * h + 1]);
          *reinterpret_cast<uint4*>(a.out + pix * COUT + 8 * c8) = o;
        }
      }
      if (a.out_f32) {
#pragma unroll
        for (int c4 = 0; c4 < COUT / 4; ++c4)
          *reinterpret_cast<float4*>(a.out_f32 + pix * COUT + 4 * c4) =
              make_float4(v[4 * c4], v[4 * c4 + 1], v[4 * c4 + 2], v[4 * c4 + 3]);
      }
    }
    // every lane's reads of accumulator b are done before tile j + 2's MMAs write it
    tc_fence_before();
    failed = __syncthreads_or((!ok || fail) ? 1 : 0) != 0;
  }
  if (failed && tid == 0) {
    atomicExch(&g_tc_error, 1);
    // copies and MMAs issued before the failure complete (bounded waits) before
    // the CTA frees its tensor memory
    auto drain = [&](unsigned long long* bar, int waited, int issued) {
      while (waited < issued && mbar_wait(smem_addr(bar), waited & 1)) ++waited;
    };
    drain(&sm.bar_tma[0], tma_w0, tma_n0);
    drain(&sm.bar_tma[1], tma_w1, tma_n1);
    drain(&sm.bar_mma[0], mma_w0, mma_n0);
    drain(&sm.bar_mma[1], mma_w1, mma_n1);
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem));
}


using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

template <int CIN, int COUT>
cudaError_t launch_tc(const ConvArgs& a, cudaStream_t s) {
  const EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // the activation tensor as (channel, x, y, image), innermost first; a box of 8
  // channels x 130 pixels x 3 rows, zero outside the tensor
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)CIN, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
  const cuuint64_t strides[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)a.W * CIN * 2, (cuuint64_t)a.H * a.W * CIN * 2};
  const cuuint32_t box[4] = {8, HP, HROWS, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(a.x), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  constexpr int smem = (int)sizeof(TcSmem<CIN, COUT>) + 1024;  // + alignment slack
  static int grid_max = 0;
  if (!grid_max) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    // all of the unified L1 / shared storage as shared memory: several CTAs per SM
    // overlap one CTA's TMA and MMAs with another's epilogue
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    // resident CTAs per SM from the SM's shared memory and registers, at most
    // 8 (each CTA holds 64 of the SM's 512 tensor-memory columns)
    int dev = 0, nsm = 148, smem_sm = 0, reserved = 0, regs_sm = 65536;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, conv3x3_tc_kernel<CIN, COUT>);
    if (e != cudaSuccess) return e;
    const int by_smem = smem_sm / (smem + (int)fa.sharedSizeBytes + reserved);
    const int by_regs = regs_sm / ((fa.numRegs > 0 ? fa.numRegs : 1) * 128);
    int per_sm = by_smem < by_regs ? by_smem : by_regs;
    per_sm = per_sm < 1 ? 1 : per_sm > 8 ? 8 : per_sm;
    grid_max = nsm * per_sm;
  }
  const int ntiles = a.B * a.H * (a.W / TP);
  const int grid = ntiles < grid_max ? ntiles : grid_max;
  conv3x3_tc_kernel<CIN, COUT><<<grid, 128, smem, s>>>(map, a, ntiles);
  return cudaGetLastError();
}

}  // namespace

bool conv3x3_tc_supported(int cin, int cout, int W) {
  return W >= TP && W % TP == 0 && (cin == 16 || cin == 32) && (cout == 16 || cout == 32) && encode_fn() != nullptr;
}

cudaError_t conv3x3_tc(int cin, int cout, const ConvArgs& a, cudaStream_t s) {
  if (a.W % TP != 0) return cudaErrorInvalidValue;
  if (cin == 16 && cout == 32) return launch_tc<16, 32>(a, s);
  if (cin == 32 && cout == 32) return launch_tc<32, 32>(a, s);
  if (cin == 32 && cout == 16) return launch_tc<32, 16>(a, s);
  return cudaErrorInvalidValue;
}

cudaError_t conv3x3_tc_error(int* flag) {
  cudaError_t e = cudaMemcpyFromSymbol(flag, g_tc_error, sizeof(int));
  if (e == cudaSuccess && *flag) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
  }
  return e;
}

}  // namespace net
}  // namespace cdm
