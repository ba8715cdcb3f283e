// Split-precision mode product on the sm_100a tensor cores (tcgen05 + TMA + TMEM).
//
// One mode product of mcc3 (src/mcc.jl:35-47: K1[n,j,k] = Σ_i Ψ[i,j,k] φ[i,n],
// and its two successors) is a GEMM
//     D[r,p] = Σ_a A[a + lda*r] * B[a + ldb*p]        r < R, p < M, a < K
// whose operands are both K-major (the contracted index is the contiguous one)
// and whose output rows are contiguous, so the output of one product is
// directly the K-major A operand of the next (the index order rotates
// [i,j,k] → [j,k,n] → [k,n,m] → [n,m,l]).
//
// Each operand is held as two planes, hi and lo, with x ≈ hi + lo:
//   kind 1: BF16 planes, tcgen05.mma.kind::f16   (BF16×3)
//   kind 2: TF32 values in FP32 planes, tcgen05.mma.kind::tf32  (TF32×3)
// and each K step issues hi·hi + hi·lo + lo·hi into one FP32 TMEM accumulator.
//
// Kernel structure (persistent, one CTA per SM; 192 threads in the 1-CTA tile,
// 192 or 320 in the CTA-pair tile, whose eight epilogue warps, where used, take
// the even and odd 32-column chunks of each TMEM lane quadrant):
//   warp 0      TMA producer: 4 tiled loads per stage (A_hi, A_lo, B_hi, B_lo),
//               128-byte swizzle, no multicast, completion on an mbarrier.
//   warp 1      TMEM allocation (512 columns = two 128×256 FP32 accumulators)
//               and the single MMA-issuing thread.
//   warps 2..5  (2..9) epilogue: tcgen05.ld of the accumulator (warp w reads TMEM lanes
//               32*(w%4)..+31), conversion to the output format (FP32, or the
//               hi/lo planes of the next product) and coalesced stores.
// Double-buffered accumulators let the epilogue of tile t overlap the MMAs of
// tile t+1.  Every mbarrier wait is bounded by a wall-clock limit; on expiry
// the CTA records an error in the device status word, drains its own copies
// and MMAs in flight, frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>

#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int BM = 128;                    // tile rows (UMMA M)
constexpr int BN_MAX = 256;                // tile modes (UMMA N upper bound)
constexpr int ROW_BYTES = 128;             // one swizzle row of K per stage
constexpr int STAGES = 2;
constexpr int A_BYTES = BM * ROW_BYTES;    // 16 KB per plane
constexpr int B_BYTES = BN_MAX * ROW_BYTES;  // 32 KB per plane
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int TMEM_COLS = 2 * BN_MAX;
constexpr int NUM_THREADS = 192;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
// Drains on the abort path (copies and MMAs already issued) always get 2 s,
// whatever the limit of the ordinary waits (TcParams::wait_ns, 2 s by
// default), so that nothing is in flight when the CTA frees TMEM and exits.
constexpr uint64_t DRAIN_NS = 2000000000ull;

struct TcParams {
    int64_t R, K, M;
    int64_t F, F_pad, ldd;
    int bn, n_tiles, m_tiles, k_chunks, elems_per_row;
    int out_kind;
    int sym;  // symmetric output (pair kernel): 1 = ModeProduct::sym, 2 = ModeProduct::sym_inner,
              // 3 = ModeProduct::sym_full
    int inner_upper;               // ModeProduct::inner_upper (with sym 2)
    int packed;                    // ModeProduct::packed (with sym 3)
    int vec;  // F, F_pad, ldd multiples of 8: 8 consecutive rows are 8 consecutive, aligned elements
    int a_mn;                      // A read MN-major through a 3-D map (ModeProduct::a_mn)
    int64_t b_group, b_group_ld;   // ModeProduct::b_group / b_group_ld (pair kernel)
    int64_t Fv;                    // rows r with r % F >= Fv are not stored
    int tma_out;                   // output stored by TMA from the staging block (pair kernel):
                                   // 1 = FP32 with outer symmetry (mD direct, mDt mirrored box),
                                   // 2 = BF16 planes with inner symmetry (mD hi, mDt lo plane)
    void* d_hi;
    void* d_lo;
    int* status;
    uint64_t wait_ns;              // limit of every ordinary mbarrier wait
};

__device__ __forceinline__ uint32_t saddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait.  Returns false (after flagging the CTA and the device status
// word) when the phase does not complete within `limit_ns`, or when another
// role of this CTA has already given up (unless `ignore_abort`, the drains,
// which always wait up to DRAIN_NS).
__device__ __noinline__ bool mbar_wait_slow(uint64_t* b, uint32_t parity, volatile int* abort_flag, int* status,
                                            int code, bool ignore_abort, uint64_t limit_ns) {
    const uint64_t t0 = gtimer();
    const uint64_t lim = ignore_abort ? DRAIN_NS : limit_ns;
    while (true) {
        if (mbar_try(b, parity)) return true;
        if (!ignore_abort && *abort_flag) return false;
        if (gtimer() - t0 > lim) {
            *abort_flag = 1;
            atomicCAS(status, 0, code);
            return false;
        }
    }
}

__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, int* status,
                                          int code, uint64_t limit_ns, bool ignore_abort = false) {
    if (mbar_try(b, parity)) return true;
    return mbar_wait_slow(b, parity, abort_flag, status, code, ignore_abort, limit_ns);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
    d |= (uint64_t)1 << 46;             // descriptor version for tcgen05
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

// Shared-memory matrix descriptor: MN-major.  Each 128-byte row holds
// consecutive M (or N) elements of one K index, and the atoms of the next 128
// bytes of M lie `lbo` bytes further on.  BF16: 128-byte swizzle of 16-byte
// chunks, 8-row K groups 1024 bytes apart.  TF32: MN-major 32-bit operands take
// the 128-byte swizzle of 32-byte chunks (layout type 1), 4-row K groups 512
// bytes apart.
template <int KIND>
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr, uint32_t lbo) {
    constexpr uint32_t sbo = KIND == 1 ? 1024u : 512u;
    constexpr uint64_t layout = KIND == 1 ? 2u : 1u;
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;  // leading byte offset: between 128-byte M atoms
    d |= (uint64_t)(sbo >> 4) << 32;             // stride byte offset: between K groups
    d |= (uint64_t)1 << 46;                      // descriptor version for tcgen05
    d |= layout << 61;
    return d;
}

// Instruction descriptor: FP32 accumulator, B K-major, A K-major or (a_mn)
// MN-major.
template <int KIND>
__device__ __forceinline__ uint32_t instr_desc(int m, int n, bool a_mn = false) {
    const uint32_t fmt = KIND == 1 ? 1u : 2u;  // BF16 : TF32
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((a_mn ? 1u : 0u) << 15) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

template <int KIND>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    if constexpr (KIND == 1) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
          "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
          "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
          "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16 TMEM lanes × 4 blocks of 8 FP32 columns in the mma accumulator fragment
// layout: thread t gets, for block k, v[4k..4k+1] = row t/4, columns
// 8k + 2(t%4) and +1, and v[4k+2..4k+3] = row t/4 + 8, the same columns.
__device__ __forceinline__ void tmem_ld_16x256b_x4(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Four 8×8 BF16 matrices from their mma fragments (register i = matrix i:
// row t/4, columns 2(t%4) and +1), each written transposed: the shared-memory
// row given by thread 8i + r receives column r of matrix i (8 rows, 16 bytes).
__device__ __forceinline__ void stmatrix_x4_trans(uint32_t addr, uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    asm volatile("stmatrix.sync.aligned.x4.trans.m8n8.shared.b16 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(r0),
                 "r"(r1), "r"(r2), "r"(r3)
                 : "memory");
}

// hi and lo BF16 planes of two FP32 values (lo = the rounding residual of hi)
__device__ __forceinline__ void split_bf16x2(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const float x = __uint_as_float(a), y = __uint_as_float(b);
    const __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(x - __uint_as_float(hi << 16), y - __uint_as_float(hi & 0xFFFF0000u));
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ float tf32_round(float v) {
    uint32_t hb;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(v));
    return __uint_as_float(hb);
}

__device__ __forceinline__ void store_one(const TcParams& p, int64_t off, float v) {
    if (p.out_kind == 0) {
        static_cast<float*>(p.d_hi)[off] = v;
    } else if (p.out_kind == 1) {
        __nv_bfloat16 h = __float2bfloat16_rn(v);
        static_cast<__nv_bfloat16*>(p.d_hi)[off] = h;
        static_cast<__nv_bfloat16*>(p.d_lo)[off] = __float2bfloat16_rn(v - __bfloat162float(h));
    } else {
        const float h = tf32_round(v);
        static_cast<float*>(p.d_hi)[off] = h;
        static_cast<float*>(p.d_lo)[off] = v - h;
    }
}

// A full chunk: this thread's row, 32 consecutive modes; element j goes to
// off + j*ldd.  Lanes of the warp hold consecutive rows, so each store
// instruction writes one contiguous segment per output plane.
template <int OUT>
__device__ __forceinline__ void store_chunk(const TcParams& p, int64_t off, const uint32_t (&v)[32]) {
    const int64_t ldd = p.ldd;
    if constexpr (OUT == 0) {
        float* d = static_cast<float*>(p.d_hi) + off;
#pragma unroll
        for (int j = 0; j < 32; ++j) d[j * ldd] = __uint_as_float(v[j]);
    } else if constexpr (OUT == 1) {
        __nv_bfloat16* dh = static_cast<__nv_bfloat16*>(p.d_hi) + off;
        __nv_bfloat16* dl = static_cast<__nv_bfloat16*>(p.d_lo) + off;
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            const float a = __uint_as_float(v[j]), b = __uint_as_float(v[j + 1]);
            const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
            const uint32_t hu = *reinterpret_cast<const uint32_t*>(&h);
            const __nv_bfloat162 l =
                __floats2bfloat162_rn(a - __uint_as_float(hu << 16), b - __uint_as_float(hu & 0xFFFF0000u));
            dh[j * ldd] = h.x;
            dh[(j + 1) * ldd] = h.y;
            dl[j * ldd] = l.x;
            dl[(j + 1) * ldd] = l.y;
        }
    } else {
        float* dh = static_cast<float*>(p.d_hi) + off;
        float* dl = static_cast<float*>(p.d_lo) + off;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float x = __uint_as_float(v[j]), h = tf32_round(x);
            dh[j * ldd] = h;
            dl[j * ldd] = x - h;
        }
    }
}

// Eight consecutive rows of one column (element offset `off`, a multiple of 8).
__device__ __forceinline__ void store_vec8(const TcParams& p, int64_t off, const float (&x)[8]) {
    if (p.out_kind == 1) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
            const uint32_t hu = *reinterpret_cast<const uint32_t*>(&hb);
            const __nv_bfloat162 lb = __floats2bfloat162_rn(x[2 * i] - __uint_as_float(hu << 16),
                                                            x[2 * i + 1] - __uint_as_float(hu & 0xFFFF0000u));
            h[i] = hu;
            l[i] = *reinterpret_cast<const uint32_t*>(&lb);
        }
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(p.d_hi) + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(p.d_lo) + off) = make_uint4(l[0], l[1], l[2], l[3]);
    } else if (p.out_kind == 0) {
        float4* d = reinterpret_cast<float4*>(static_cast<float*>(p.d_hi) + off);
        d[0] = make_float4(x[0], x[1], x[2], x[3]);
        d[1] = make_float4(x[4], x[5], x[6], x[7]);
    } else {
        float hv[8], lv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            hv[i] = tf32_round(x[i]);
            lv[i] = x[i] - hv[i];
        }
        float4* dh = reinterpret_cast<float4*>(static_cast<float*>(p.d_hi) + off);
        float4* dl = reinterpret_cast<float4*>(static_cast<float*>(p.d_lo) + off);
        dh[0] = make_float4(hv[0], hv[1], hv[2], hv[3]);
        dh[1] = make_float4(hv[4], hv[5], hv[6], hv[7]);
        dl[0] = make_float4(lv[0], lv[1], lv[2], lv[3]);
        dl[1] = make_float4(lv[4], lv[5], lv[6], lv[7]);
    }
}

// Symmetric output: does pair tile (mt, nt) hold any column >= its rows' outer
// index (sym 1), or any column >= its rows' inner index (sym 2: the 256 rows of
// a tile share one outer index and the tiles are square)?  With full symmetry
// (sym 3) a row tile is computed, every column of it, when T(a) <= T(b); with
// the packed output only its mode tiles that reach s >= b.
__device__ __forceinline__ bool sym_tile_live(const TcParams& p, int mt, int nt) {
    if (p.sym == 3) {
        const int64_t r0 = (int64_t)mt * 256, a0 = r0 % p.F, b = r0 / p.F;
        if (p.packed) {  // only entries a <= b <= s are stored
            int64_t smax = (int64_t)nt * p.bn + p.bn;
            if (smax > p.M) smax = p.M;
            return a0 <= b && smax - 1 >= b;
        }
        return a0 / 256 <= b / 256;
    }
    const int64_t pmin = p.sym == 2 ? ((int64_t)mt * 256) % p.F : ((int64_t)mt * 256) / p.F;
    int64_t qmax = (int64_t)nt * p.bn + p.bn;
    if (qmax > p.M) qmax = p.M;
    return qmax - 1 >= pmin;
}

// TMA store of a box from this CTA's shared memory (bulk-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z), "r"(saddr(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The staging block may be written again once the TMA engine has read it.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Transposed stores of one 32 × 32 block (inner symmetry): element (row r,
// column c0 + j) goes to (c0 + j) + F_pad·(r / F) + ldd·(r % F), so the columns
// of a row are contiguous.  Each lane packs its own row (v[j], j < 32) into the
// warp's staging block — 16-byte chunks XOR-swizzled by row so that neither
// the writes nor the reads conflict — and the warp then stores whole row
// segments: 8 rows × 64 bytes (BF16) or 4 rows × 128 bytes (TF32, one plane
// after the other) per instruction.  The output planes are of the operand
// kind (the host requires out_kind == KIND with inner symmetry).  Rows whose inner index is not below M
// (padding) and columns past `ncols` are not stored.
// The warp's 32 rows lie in one block of F rows: outer index pk, inner indices
// pp0 + row.
template <int KIND>
__device__ __forceinline__ void mirror_rows(const TcParams& p, uint8_t* sb, const uint32_t (&v)[32], int lane,
                                            int64_t pk, int64_t pp0, int64_t c0, int64_t ncols,
                                            const CUtensorMap* md, const CUtensorMap* mdt) {
    const int64_t base = c0 + p.F_pad * pk + p.ldd * pp0;
    if constexpr (KIND == 1) {
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint32_t h[4], l[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float a = __uint_as_float(v[8 * g + 2 * i]), b = __uint_as_float(v[8 * g + 2 * i + 1]);
                const __nv_bfloat162 hb = __floats2bfloat162_rn(a, b);
                const uint32_t hu = *reinterpret_cast<const uint32_t*>(&hb);
                const __nv_bfloat162 lb =
                    __floats2bfloat162_rn(a - __uint_as_float(hu << 16), b - __uint_as_float(hu & 0xFFFF0000u));
                h[i] = hu;
                l[i] = *reinterpret_cast<const uint32_t*>(&lb);
            }
            const int sw = g ^ ((lane >> 1) & 3);
            *reinterpret_cast<uint4*>(sb + lane * 64 + sw * 16) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(sb + 2048 + lane * 64 + sw * 16) = make_uint4(l[0], l[1], l[2], l[3]);
        }
        if (p.tma_out == 2 && (ncols == 32 || c0 + ncols == p.M)) {
            // the staging rows are the 64-byte-swizzled box (columns × 1 × rows)
            // of the planes' map: rows past M and columns past the matrix are
            // clipped by the map
            if (pp0 >= p.M) return;  // padding rows only
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
                tma_store_3d(md, sb, (int)c0, (int)pk, (int)pp0);
                tma_store_3d(mdt, sb + 2048, (int)c0, (int)pk, (int)pp0);
                bulk_commit();
            }
            __syncwarp();
            return;
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = 8 * i + (lane >> 2), c = lane & 3, sw = c ^ ((row >> 1) & 3);
            const uint4 vh = *reinterpret_cast<const uint4*>(sb + row * 64 + sw * 16);
            const uint4 vl = *reinterpret_cast<const uint4*>(sb + 2048 + row * 64 + sw * 16);
            if (pp0 + row < p.M && 8 * c < ncols) {
                const int64_t off = base + 8 * c + p.ldd * row;
                *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(p.d_hi) + off) = vh;
                *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(p.d_lo) + off) = vl;
            }
        }
    } else {
#pragma unroll
        for (int plane = 0; plane < 2; ++plane) {
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                float x[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float a = __uint_as_float(v[4 * g + i]), hv = tf32_round(a);
                    x[i] = plane == 0 ? hv : a - hv;
                }
                const int sw = g ^ (lane & 7);
                *reinterpret_cast<float4*>(sb + lane * 128 + sw * 16) = make_float4(x[0], x[1], x[2], x[3]);
            }
            __syncwarp();
            float* dst = static_cast<float*>(plane == 0 ? p.d_hi : p.d_lo);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int row = 4 * i + (lane >> 3), c = lane & 7, sw = c ^ (row & 7);
                const float4 y = *reinterpret_cast<const float4*>(sb + row * 128 + sw * 16);
                if (pp0 + row < p.M && 4 * c < ncols)
                    *reinterpret_cast<float4*>(dst + base + 4 * c + p.ldd * row) = y;
            }
            __syncwarp();
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    mode_product_tc_kernel(const __grid_constant__ CUtensorMap mA_hi, const __grid_constant__ CUtensorMap mA_lo,
                           const __grid_constant__ CUtensorMap mB_hi, const __grid_constant__ CUtensorMap mB_lo,
                           const TcParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;
    uint64_t* tempty = tfull + 2;
    uint64_t* drain = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 128);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int total = p.m_tiles * p.n_tiles;

    if (warp == 0) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer
            int stage = 0;
            uint32_t phase = 0;
            uint32_t filled = 0, filled_phase = 0;  // per-stage bit masks
            bool ok = true;
            const uint32_t tx = 2u * A_BYTES + 2u * (uint32_t)p.bn * ROW_BYTES;
            for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
                const int nt = t % p.n_tiles, mt = t / p.n_tiles;
                for (int kc = 0; kc < p.k_chunks; ++kc) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.status, DEV_TIMEOUT_PRODUCER, p.wait_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t* st = smem + stage * STAGE_BYTES;
                    mbar_expect_tx(&full[stage], tx);
                    const int x = kc * p.elems_per_row;
                    tma_load_2d(st, &mA_hi, &full[stage], x, mt * BM);
                    tma_load_2d(st + A_BYTES, &mA_lo, &full[stage], x, mt * BM);
                    tma_load_2d(st + 2 * A_BYTES, &mB_hi, &full[stage], x, nt * p.bn);
                    tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mB_lo, &full[stage], x, nt * p.bn);
                    filled |= 1u << stage;
                    filled_phase = (filled_phase & ~(1u << stage)) | (phase << stage);
                    if (++stage == STAGES) stage = 0, phase ^= 1;
                }
            }
            if (!ok || *abort_flag) {
                // Let the copies already issued land before the CTA exits.
                for (int s = 0; s < STAGES; ++s)
                    if (filled & (1u << s))
                        mbar_wait(&full[s], (filled_phase >> s) & 1u, abort_flag, p.status, DEV_TIMEOUT_PRODUCER,
                                  p.wait_ns, true);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ------------------------------------------------ MMA issuer
            const uint32_t idesc = instr_desc<KIND>(BM, p.bn);
            int stage = 0, acc = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true, issued = false;
            for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
                if (!mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN_MAX);
                for (int kc = 0; kc < p.k_chunks; ++kc) {
                    if (!mbar_wait(&full[stage], phase, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t base = saddr(smem + stage * STAGE_BYTES);
                    const uint64_t a_hi = smem_desc(base), a_lo = smem_desc(base + A_BYTES);
                    const uint64_t b_hi = smem_desc(base + 2 * A_BYTES);
                    const uint64_t b_lo = smem_desc(base + 2 * A_BYTES + B_BYTES);
#pragma unroll
                    for (int k = 0; k < ROW_BYTES / 32; ++k) {
                        const uint64_t off = (uint64_t)((k * 32) >> 4);
                        umma<KIND>(d_tmem, a_hi + off, b_hi + off, idesc, (kc | k) != 0);
                        umma<KIND>(d_tmem, a_hi + off, b_lo + off, idesc, 1u);
                        umma<KIND>(d_tmem, a_lo + off, b_hi + off, idesc, 1u);
                    }
                    umma_commit(&empty[stage]);
                    issued = true;
                    if (++stage == STAGES) stage = 0, phase ^= 1;
                }
                if (!ok) break;
                umma_commit(&tfull[acc]);
                if (++acc == 2) acc = 0, acc_phase ^= 1;
            }
            if ((!ok || *abort_flag) && issued) {
                // Wait for every MMA this thread issued before TMEM is freed.
                umma_commit(drain);
                mbar_wait(drain, 0, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns, true);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------- epilogue
        const int q = warp & 3;  // TMEM lane quadrant this warp may access
        int acc = 0;
        uint32_t acc_phase = 0;
        const int chunks = (p.bn + 31) / 32;
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            const int nt = t % p.n_tiles, mt = t / p.n_tiles;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&tfull[acc], acc_phase, abort_flag, p.status, DEV_TIMEOUT_EPILOGUE, p.wait_ns);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            tc_fence_after();
            const int64_t row = (int64_t)mt * BM + q * 32 + lane;
            const bool row_ok = row < p.R;
            const int64_t row_off = row_ok ? (row % p.F) + p.F_pad * (row / p.F) : 0;
            const int64_t col0 = (int64_t)nt * p.bn;
            for (int ch = 0; ch < chunks; ++ch) {
                uint32_t v[32];
                tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN_MAX + ch * 32), v);
                if (!row_ok) continue;
                const int64_t c0 = col0 + ch * 32;
                const int64_t off = row_off + p.ldd * c0;
                if (ch * 32 + 32 <= p.bn && c0 + 32 <= p.M) {
                    if (p.out_kind == 1)
                        store_chunk<1>(p, off, v);
                    else if (p.out_kind == 0)
                        store_chunk<0>(p, off, v);
                    else
                        store_chunk<2>(p, off, v);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (ch * 32 + j < p.bn && c0 + j < p.M) store_one(p, off + p.ldd * j, __uint_as_float(v[j]));
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            if (++acc == 2) acc = 0, acc_phase ^= 1;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// 2-CTA variant (cta_group::2).  A cluster of two CTAs computes a tile of 256
// rows × up to 256 modes: each CTA stages its own 128 rows of the operand and
// its half of the φ mode tile, the leader (cluster rank 0) issues
// tcgen05.mma.cta_group::2 (M = 256) reading both CTAs' shared memory, and
// each CTA's TMEM receives its 128 rows of the accumulator.  Per SM this moves
// half as many φ bytes per flop as the 1-CTA tile.  The peer's TMA loads
// complete on the leader's mbarrier (cp.async.bulk.tensor .cta_group::2, no
// multicast); the leader's commits multicast to both CTAs' barriers to free
// their stages and to start both epilogues; the epilogue warps of both CTAs
// arrive on the leader's accumulator-empty barrier.
constexpr int STAGES2 = 3;
constexpr int B2_BYTES = (BN_MAX / 2) * ROW_BYTES;       // half of the mode tile, one plane
constexpr int STAGE2_BYTES = 2 * A_BYTES + 2 * B2_BYTES;
// Epilogue warps after the TMA-producer and MMA-issuer warps: 4 (one per TMEM
// lane quadrant) or 8 (two per quadrant, even and odd 32-column chunks).  The
// grouped second product, whose K is short, takes 8; the others take 4, which
// leaves room on every SM for the FP64 Ψ writer running beside them.
template <int EPI>
constexpr int pair_threads() { return 32 * (2 + EPI); }
// Epilogue staging: per epilogue warp a 32-column × 32-row FP32 block stored by
// column (rows contiguous); the two 16-byte halves of every 8-row group swap
// places in odd columns, so that the writes by row and the 128-bit reads by
// column are both free of bank conflicts.
constexpr int STG_LD = 32;
template <int EPI>
constexpr int pair_smem_bytes() { return STAGES2 * STAGE2_BYTES + 1024 + 256 + EPI * 32 * STG_LD * 4; }
static_assert(pair_smem_bytes<8>() <= 232448, "pair-kernel shared memory over the 227 KB limit");

__device__ __forceinline__ int stg_idx(int col, int row) { return col * STG_LD + (row ^ ((col & 1) << 2)); }

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster, int x,
                                                 int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster, int x,
                                                 int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3, %4}], [%5];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar_cluster)
        : "memory");
}

template <int KIND>
__device__ __forceinline__ void umma_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    if constexpr (KIND == 1) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    }
}

// arrive on the barrier at this address in both CTAs of the pair
__device__ __forceinline__ void umma_commit_pair_both(uint64_t* bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            saddr(bar)),
        "h"(mask)
        : "memory");
}

__device__ __forceinline__ void umma_commit_pair_own(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// Cancels `bytes` of the current phase's expected transaction count.
__device__ __forceinline__ void mbar_complete_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint32_t ld_shared_cluster_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

// 128 registers at most: the register file is split over the SM's four
// partitions, and two 256-thread blocks of the FP64 Ψ writer (64 registers)
// fit beside the six warps of the 4-epilogue-warp form only at that size.
template <int KIND, int EPI>
__global__ void __maxnreg__(128)
    mode_product_tc2_kernel(const __grid_constant__ CUtensorMap mA_hi, const __grid_constant__ CUtensorMap mA_lo,
                            const __grid_constant__ CUtensorMap mB_hi, const __grid_constant__ CUtensorMap mB_lo,
                            const __grid_constant__ CUtensorMap mD, const __grid_constant__ CUtensorMap mDt,
                            const TcParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    // operand stages, then the epilogue staging blocks (1024-byte aligned, as
    // the TMA store's 128-byte swizzle wants), then the barriers
    float* stage_base = reinterpret_cast<float*>(smem + STAGES2 * STAGE2_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES2 * STAGE2_BYTES + EPI * 32 * STG_LD * 4);
    uint64_t* empty = full + STAGES2;
    uint64_t* tfull = empty + STAGES2;
    uint64_t* tempty = tfull + 2;
    uint64_t* drain = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    uint32_t* nfill = reinterpret_cast<uint32_t*>(tmem_slot + 2);  // loads issued per stage (this CTA)

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES2; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * EPI);  // the epilogue warps of both CTAs
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        for (int st = 0; st < STAGES2; ++st) nfill[st] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int total = p.m_tiles * p.n_tiles;
    const int half = p.bn / 2;

    if (warp == 0) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer (both CTAs)
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            const uint32_t tx_pair = 2u * (2u * A_BYTES + 2u * (uint32_t)half * ROW_BYTES);
            for (int t = pair; t < total && ok; t += npairs) {
                const int nt = t % p.n_tiles, mt = t / p.n_tiles;
                if (p.sym && !sym_tile_live(p, mt, nt)) continue;
                for (int kc = 0; kc < p.k_chunks; ++kc) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.status, DEV_TIMEOUT_PRODUCER, p.wait_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t* st = smem + stage * STAGE2_BYTES;
                    const uint32_t fb = mapa_shared(saddr(&full[stage]), 0);
                    if (leader) mbar_expect_tx(&full[stage], tx_pair);
                    const int x = kc * p.elems_per_row;
                    const int64_t row0 = (int64_t)mt * 256 + (int)rank * 128;
                    if (p.a_mn) {
                        // 128 rows = (128 / epr) boxes of epr M-elements × epr K-rows
                        const int z = (int)(row0 / p.F), m0 = (int)(row0 % p.F);
                        for (int i = 0; i < 128 / p.elems_per_row; ++i) {
                            const int off = i * p.elems_per_row * ROW_BYTES;
                            tma_load_3d_pair(st + off, &mA_hi, fb, m0 + i * p.elems_per_row, x, z);
                            tma_load_3d_pair(st + A_BYTES + off, &mA_lo, fb, m0 + i * p.elems_per_row, x, z);
                        }
                    } else {
                        tma_load_2d_pair(st, &mA_hi, fb, x, (int)row0);
                        tma_load_2d_pair(st + A_BYTES, &mA_lo, fb, x, (int)row0);
                    }
                    const int by = nt * p.bn + (int)rank * half +
                                   (p.b_group ? (int)(((int64_t)mt * 256 / p.b_group) * p.b_group_ld) : 0);
                    tma_load_2d_pair(st + 2 * A_BYTES, &mB_hi, fb, x, by);
                    tma_load_2d_pair(st + 2 * A_BYTES + B2_BYTES, &mB_lo, fb, x, by);
                    ++nfill[stage];
                    if (++stage == STAGES2) stage = 0, phase ^= 1;
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ------------------------------------------------ MMA issuer (leader)
            const uint32_t idesc = instr_desc<KIND>(256, p.bn, p.a_mn != 0);
            // MN-major A: one UMMA K step (32 bytes of K) is 32/esz K-rows of 128 bytes
            const uint32_t a_step = p.a_mn ? (uint32_t)(32 / (KIND == 1 ? 2 : 4)) * ROW_BYTES : 32u;
            const uint32_t a_lbo = (uint32_t)p.elems_per_row * ROW_BYTES;
            int stage = 0, acc = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true, issued = false;
            for (int t = pair; t < total && ok; t += npairs) {
                if (p.sym && !sym_tile_live(p, t / p.n_tiles, t % p.n_tiles)) continue;
                if (!mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN_MAX);
                for (int kc = 0; kc < p.k_chunks; ++kc) {
                    if (!mbar_wait(&full[stage], phase, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t base = saddr(smem + stage * STAGE2_BYTES);
                    const uint64_t a_hi = p.a_mn ? smem_desc_mn<KIND>(base, a_lbo) : smem_desc(base);
                    const uint64_t a_lo =
                        p.a_mn ? smem_desc_mn<KIND>(base + A_BYTES, a_lbo) : smem_desc(base + A_BYTES);
                    const uint64_t b_hi = smem_desc(base + 2 * A_BYTES);
                    const uint64_t b_lo = smem_desc(base + 2 * A_BYTES + B2_BYTES);
#pragma unroll
                    for (int k = 0; k < ROW_BYTES / 32; ++k) {
                        const uint64_t off = (uint64_t)((k * 32) >> 4);
                        const uint64_t aoff = (uint64_t)((k * a_step) >> 4);
                        umma_pair<KIND>(d_tmem, a_hi + aoff, b_hi + off, idesc, (kc | k) != 0);
                        umma_pair<KIND>(d_tmem, a_hi + aoff, b_lo + off, idesc, 1u);
                        umma_pair<KIND>(d_tmem, a_lo + aoff, b_hi + off, idesc, 1u);
                    }
                    umma_commit_pair_both(&empty[stage]);
                    issued = true;
                    if (++stage == STAGES2) stage = 0, phase ^= 1;
                }
                if (!ok) break;
                umma_commit_pair_both(&tfull[acc]);
                if (++acc == 2) acc = 0, acc_phase ^= 1;
            }
            if ((!ok || *abort_flag) && issued) {
                umma_commit_pair_own(drain);
                mbar_wait(drain, 0, abort_flag, p.status, DEV_TIMEOUT_MMA, p.wait_ns, true);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------- epilogue (both CTAs)
        const int q = warp & 3;             // TMEM lane quadrant this warp may access
        const int cpar = (warp - 2) >> 2;   // with 8 epilogue warps: even (0) or odd (1) 32-column chunks
        int acc = 0;
        uint32_t acc_phase = 0;
        const int chunks = (p.bn + 31) / 32;
        for (int t = pair; t < total; t += npairs) {
            const int nt = t % p.n_tiles, mt = t / p.n_tiles;
            if (p.sym && !sym_tile_live(p, mt, nt)) continue;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&tfull[acc], acc_phase, abort_flag, p.status, DEV_TIMEOUT_EPILOGUE, p.wait_ns);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            tc_fence_after();
            const int64_t row = (int64_t)mt * 256 + rank * 128 + q * 32 + lane;
            const bool row_ok = row < p.R && (row % p.F) < p.Fv;
            const int64_t row_off = row_ok ? (row % p.F) + p.F_pad * (row / p.F) : 0;
            const int64_t col0 = (int64_t)nt * p.bn;
            const int64_t wrow0 = (int64_t)mt * 256 + rank * 128 + q * 32;  // the warp's first row
            const bool warp_vec = p.vec && wrow0 + 32 <= p.R;
            // sym 2: a tile wholly above the diagonal is also stored transposed
            const bool sym2_mirror =
                p.sym == 2 && !p.inner_upper && (int64_t)nt * p.bn >= ((int64_t)mt * 256) % p.F + 256;
            float* stg = stage_base + (warp - 2) * (32 * STG_LD);
            for (int ch = cpar; ch < chunks; ch += EPI / 4) {
                if constexpr (KIND == 1) {
                    if (p.tma_out == 2 && warp_vec) {
                        // BF16 planes by TMA (inner symmetry), staged through stmatrix:
                        // the accumulator is read in the mma fragment layout (two
                        // 16-lane halves), packed to hi/lo BF16 pairs, and each 8×8
                        // block is written transposed into the 64-byte-swizzled
                        // [column][row] staging of the box, 16 bytes per row.
                        const int64_t c0 = col0 + ch * 32;
                        int64_t ncols = p.M - c0;
                        if (ncols > p.bn - ch * 32) ncols = p.bn - ch * 32;
                        if (ncols > 32) ncols = 32;
                        if (ncols > 0 && (ncols == 32 || c0 + ncols == p.M)) {
                            const int64_t pk = wrow0 / p.F, pp0 = wrow0 - pk * p.F;
                            uint32_t f0[16], f1[16];
                            const uint32_t tcol = (uint32_t)(acc * BN_MAX + ch * 32);
                            tmem_ld_16x256b_x4(tmem_base + ((uint32_t)(q * 32) << 16) + tcol, f0);
                            tmem_ld_16x256b_x4(tmem_base + ((uint32_t)(q * 32 + 16) << 16) + tcol, f1);
                            tmem_wait_ld();
                            if (lane == 0) bulk_wait_read();  // the staging block is free again
                            __syncwarp();
                            const uint32_t sbase = saddr(stg);
                            const int mi = lane >> 3, rr = lane & 7;  // this thread's matrix and row address
#pragma unroll
                            for (int g = 0; g < 4; ++g) {
                                // matrices i = 0..3: rows 8i..8i+7 of the warp, columns 8g..8g+7
                                uint32_t h0, l0, h1, l1, h2, l2, h3, l3;
                                split_bf16x2(f0[4 * g], f0[4 * g + 1], h0, l0);
                                split_bf16x2(f0[4 * g + 2], f0[4 * g + 3], h1, l1);
                                split_bf16x2(f1[4 * g], f1[4 * g + 1], h2, l2);
                                split_bf16x2(f1[4 * g + 2], f1[4 * g + 3], h3, l3);
                                const int j = 8 * g + rr;  // staging line (column)
                                const uint32_t addr = sbase + (uint32_t)(j * 64 + (((mi ^ (j >> 1)) & 3) << 4));
                                stmatrix_x4_trans(addr, h0, h1, h2, h3);
                                stmatrix_x4_trans(addr + 2048, l0, l1, l2, l3);
                            }
                            fence_proxy_async_smem();
                            __syncwarp();
                            if (lane == 0) {
                                tma_store_3d(&mD, stg, (int)pp0, (int)pk, (int)c0);
                                tma_store_3d(&mDt, reinterpret_cast<uint8_t*>(stg) + 2048, (int)pp0, (int)pk, (int)c0);
                                bulk_commit();
                            }
                            __syncwarp();
                            continue;
                        }
                        if (ncols <= 0) continue;
                        // any other partial chunk takes the general path below
                    }
                }
                uint32_t v[32];
                tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN_MAX + ch * 32), v);
                const int64_t c0 = col0 + ch * 32;
                int64_t ncols = p.M - c0;  // valid columns of this chunk
                if (ncols > p.bn - ch * 32) ncols = p.bn - ch * 32;
                if (ncols > 32) ncols = 32;
                if (p.tma_out) {
                    // the staging block may still be read by this warp's last TMA store
                    if (lane == 0) bulk_wait_read();
                    __syncwarp();
                }
                // a 32-column box may run past the last column of the matrix (the
                // map clips it) but not into the next mode tile's columns
                if constexpr (KIND == 1) {
                    if (p.tma_out == 2 && warp_vec && ncols > 0 && (ncols == 32 || c0 + ncols == p.M)) {
                        // BF16 planes by TMA (inner symmetry): [column][row], 64-byte
                        // lines, 16-byte chunks XOR-swizzled by line pair; every entry
                        // of a live tile is a direct store
                        const int64_t pk = wrow0 / p.F, pp0 = wrow0 - pk * p.F;
                        uint8_t* sb = reinterpret_cast<uint8_t*>(stg);
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const float x = __uint_as_float(v[j]);
                            const __nv_bfloat16 hb = __float2bfloat16_rn(x);
                            const __nv_bfloat16 lb = __float2bfloat16_rn(x - __bfloat162float(hb));
                            const int off = j * 64 + ((((lane >> 3) ^ (j >> 1)) & 3) << 4) + (lane & 7) * 2;
                            *reinterpret_cast<__nv_bfloat16*>(sb + off) = hb;
                            *reinterpret_cast<__nv_bfloat16*>(sb + 2048 + off) = lb;
                        }
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) {
                            tma_store_3d(&mD, sb, (int)pp0, (int)pk, (int)c0);
                            tma_store_3d(&mDt, sb + 2048, (int)pp0, (int)pk, (int)c0);
                            bulk_commit();
                        }
                        __syncwarp();
                        continue;
                    }
                }
                if (p.sym == 3) {
                    // Full symmetry: the warp's 32 rows a0.. share b, the chunk's
                    // columns share T(s); which images to store is decided per
                    // block (the host guarantees FP32 TMA output and 8-aligned
                    // shapes, and the boxes are clipped at M by the map).
                    const int64_t b = wrow0 / p.F, a0 = wrow0 - b * p.F;
                    if (ncols <= 0 || a0 >= p.Fv) continue;  // no columns, or padding rows only
                    if (p.packed) {
                        // only a <= b <= s, each entry once: for column s the run a = 0..b
                        // sits at s(s+1)(s+2)/6 + b(b+1)/2, so a warp's store of one column
                        // is 32 consecutive floats (fewer where the run ends at b)
                        if (a0 > b || c0 + ncols <= b) continue;
                        const int64_t a = a0 + lane;
                        float* dst = static_cast<float*>(p.d_hi) + b * (b + 1) / 2 + a;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int64_t sc = c0 + j;
                            if (j < ncols && sc >= b && a <= b) dst[sc * (sc + 1) * (sc + 2) / 6] = __uint_as_float(v[j]);
                        }
                        continue;
                    }
                    const int64_t ta = a0 >> 8, tb = b >> 8, ts = c0 >> 8;
                    // [s][a] lines: the direct box (a, b, s) and, when T(s) < T(a), the mirrored (a, s, b)
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        stg[j * 32 + ((((lane >> 2) ^ j) & 7) << 2) + (lane & 3)] = __uint_as_float(v[j]);
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0) {
                        tma_store_3d(&mD, stg, (int)a0, (int)b, (int)c0);
                        if (ts < ta) tma_store_3d(&mDt, stg, (int)a0, (int)c0, (int)b);
                        bulk_commit();
                    }
                    __syncwarp();
                    if (ts > tb) {
                        // [a][s] lines (each lane its own row, 16-byte chunks swizzled by
                        // line): the transposed images (s, a, b) and, when T(b) > T(a), (s, b, a)
                        if (lane == 0) bulk_wait_read();
                        __syncwarp();
                        float* line = stg + lane * 32;
#pragma unroll
                        for (int g = 0; g < 8; ++g)
                            *reinterpret_cast<float4*>(line + ((g ^ (lane & 7)) << 2)) =
                                make_float4(__uint_as_float(v[4 * g]), __uint_as_float(v[4 * g + 1]),
                                            __uint_as_float(v[4 * g + 2]), __uint_as_float(v[4 * g + 3]));
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) {
                            tma_store_3d(&mDt, stg, (int)c0, (int)a0, (int)b);
                            if (tb > ta) tma_store_3d(&mD, stg, (int)c0, (int)b, (int)a0);
                            bulk_commit();
                        }
                        __syncwarp();
                    }
                    continue;
                }
                if (p.tma_out == 1 && warp_vec && ncols > 0 && (ncols == 32 || c0 + ncols == p.M)) {
                    // FP32 output by TMA: the warp's 32 rows share one outer index
                    // pr; a chunk goes whole when every column lies on one side of
                    // the symmetric diagonal, else by the vector path below
                    const int64_t pr = wrow0 / p.F, kr0 = wrow0 - pr * p.F;
                    if (kr0 >= p.Fv) continue;  // padding rows only: nothing is stored
                    const bool d_all = !p.sym || c0 >= pr, d_none = p.sym && c0 + ncols <= pr;
                    const bool m_all = p.sym && c0 > pr, m_none = !p.sym || c0 + ncols <= pr + 1;
                    if ((d_all || d_none) && (m_all || m_none)) {
                        if (!d_none || !m_none) {
                            // [column][row], 128-byte lines, 16-byte chunks XOR-swizzled by line
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                stg[j * 32 + ((((lane >> 2) ^ j) & 7) << 2) + (lane & 3)] = __uint_as_float(v[j]);
                            fence_proxy_async_smem();
                            __syncwarp();
                            if (lane == 0) {
                                if (!d_none) tma_store_3d(&mD, stg, (int)kr0, (int)pr, (int)c0);
                                if (!m_none) tma_store_3d(&mDt, stg, (int)kr0, (int)c0, (int)pr);
                                bulk_commit();
                            }
                            __syncwarp();
                        }
                        continue;
                    }
                }
                if (warp_vec && ncols > 0) {
                    // Transpose the 32×32 block through shared memory so that each
                    // lane stores 8 consecutive rows of one column as one vector.
#pragma unroll
                    for (int j = 0; j < 32; ++j) stg[stg_idx(j, lane)] = __uint_as_float(v[j]);
                    __syncwarp();
                    const int m = lane & 3;
                    const int64_t r0 = wrow0 + 8 * m;
                    const int64_t pr = r0 / p.F, kr = r0 - pr * p.F;
                    const bool kr_ok = kr < p.Fv;  // 8-row groups are all valid or all not (Fv % 8 == 0)
#pragma unroll
                    for (int rd = 0; rd < 4; ++rd) {
                        const int j = 8 * rd + (lane >> 2);
                        if (j >= ncols || !kr_ok) continue;
                        const float4 a = *reinterpret_cast<const float4*>(stg + stg_idx(j, 8 * m));
                        const float4 b = *reinterpret_cast<const float4*>(stg + stg_idx(j, 8 * m + 4));
                        const float x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
                        const int64_t qq = c0 + j;
                        if (p.sym != 1 || qq >= pr) store_vec8(p, kr + p.F_pad * pr + p.ldd * qq, x);
                        if (p.sym == 1 && qq > pr) store_vec8(p, kr + p.F_pad * qq + p.ldd * pr, x);
                    }
                    __syncwarp();
                    continue;
                }
                if (!row_ok) continue;
                const int64_t off = row_off + p.ldd * c0;
                if (p.sym) {
                    // direct entries with column q >= p, mirrored ones (k, q, p) with q > p
                    const int64_t pr = row / p.F, kr = row - pr * p.F;
                    const int64_t moff = kr + p.ldd * pr + p.F_pad * c0;
                    const int64_t dlo = pr - c0, mlo = pr + 1 - c0;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        if (ch * 32 + j < p.bn && c0 + j < p.M) {
                            const float x = __uint_as_float(v[j]);
                            if (j >= dlo) store_one(p, off + p.ldd * j, x);
                            if (j >= mlo) store_one(p, moff + p.F_pad * j, x);
                        }
                    }
                } else if (ch * 32 + 32 <= p.bn && c0 + 32 <= p.M) {
                    if (p.out_kind == 1)
                        store_chunk<1>(p, off, v);
                    else if (p.out_kind == 0)
                        store_chunk<0>(p, off, v);
                    else
                        store_chunk<2>(p, off, v);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (ch * 32 + j < p.bn && c0 + j < p.M) store_one(p, off + p.ldd * j, __uint_as_float(v[j]));
                }
            }
            if (sym2_mirror && warp_vec) {
                // the transposed copy, a second pass over the accumulator
                // (kept apart from the direct stores to bound register use)
                for (int ch = cpar; ch < chunks; ch += EPI / 4) {
                    const int64_t c0 = col0 + ch * 32;
                    int64_t ncols = p.M - c0;
                    if (ncols > p.bn - ch * 32) ncols = p.bn - ch * 32;
                    if (ncols > 32) ncols = 32;
                    if (ncols <= 0) break;
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN_MAX + ch * 32), v);
                    if (p.tma_out) {
                        if (lane == 0) bulk_wait_read();
                        __syncwarp();
                    }
                    mirror_rows<KIND>(p, reinterpret_cast<uint8_t*>(stg), v, lane, wrow0 / p.F, wrow0 % p.F, c0,
                                      ncols, &mD, &mDt);
                    __syncwarp();
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(mapa_shared(saddr(&tempty[acc]), 0));
            if (++acc == 2) acc = 0, acc_phase ^= 1;
        }
        if (p.tma_out && lane == 0) bulk_wait_all();  // this warp's TMA stores complete
        __syncwarp();
    }

    tc_fence_before();
    cluster_sync_all();
    // Every operand load either CTA issued completes on the leader's full
    // barriers, and after an abort the two producers may have stopped one load
    // apart on a stage (each needs the other's previous load of the stage
    // consumed before issuing the next, so the counts differ by at most one).
    // The leader settles the last phase of every stage — arming a phase only
    // the peer loaded, or cancelling the peer's half of a phase only the leader
    // loaded — and waits for it (DRAIN_NS), so that no load is in flight when
    // either CTA exits.  In a run without abort the counts agree and every
    // phase has long completed.
    if (leader && threadIdx.x == 0) {
        const uint32_t peer_bytes = 2u * A_BYTES + 2u * (uint32_t)half * ROW_BYTES;
        for (int s = 0; s < STAGES2; ++s) {
            const uint32_t L = nfill[s], P = ld_shared_cluster_u32(mapa_shared(saddr(&nfill[s]), 1));
            if (L == 0 && P == 0) continue;
            if (P == L + 1) mbar_expect_tx(&full[s], peer_bytes);
            else if (L == P + 1) mbar_complete_tx(&full[s], peer_bytes);
            const uint32_t last = (L > P ? L : P) - 1;
            mbar_wait(&full[s], last & 1u, abort_flag, p.status, DEV_TIMEOUT_PRODUCER, p.wait_ns, true);
        }
    }
    cluster_sync_all();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS)
                     : "memory");
    }
}

using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(ptr);
    }
    return fn;
}

int make_map(CUtensorMap* m, const void* base, int kind, int64_t K, int64_t rows, int64_t ld, int box_rows) {
    EncodeFn enc = encode_fn();
    if (!enc) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const int esz = kind == 1 ? 2 : 4;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (ld * esz) % 16 != 0)
        return set_error(FCB_ERR_ARG, "split operand is not 16-byte aligned (padded leading dimension required)");
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * esz)};
    cuuint32_t box[2] = {(cuuint32_t)(ROW_BYTES / esz), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, kind == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                     const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return FCB_OK;
}

// 3-D map of an MN-major operand: element (m, k, z) at m + ld1·k + ld2·z; box
// of 128 bytes of m × epr k-rows × 1, swizzled as the MN-major descriptor of
// the kind expects (16-byte chunks for BF16, 32-byte chunks for TF32).
int make_map_mn(CUtensorMap* m, const void* base, int kind, int64_t Mx, int64_t K, int64_t Z, int64_t ld1,
                int64_t ld2) {
    EncodeFn enc = encode_fn();
    if (!enc) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const int esz = kind == 1 ? 2 : 4;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (ld1 * esz) % 16 != 0 || (ld2 * esz) % 16 != 0)
        return set_error(FCB_ERR_ARG, "MN-major operand is not 16-byte aligned");
    const cuuint32_t epr = (cuuint32_t)(ROW_BYTES / esz);
    cuuint64_t dims[3] = {(cuuint64_t)Mx, (cuuint64_t)K, (cuuint64_t)Z};
    cuuint64_t strides[2] = {(cuuint64_t)(ld1 * esz), (cuuint64_t)(ld2 * esz)};
    cuuint32_t box[3] = {epr, epr, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, kind == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                     const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     kind == 1 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return FCB_OK;
}

// 3-D map of an FP32 output D[(r % F) + F_pad·(r / F) + ldd·c] as (row in
// block, block, column), boxes of 32 rows × 32 blocks × 1 column or 32 rows ×
// 1 block × 32 columns, staged in shared memory as 128-byte lines with the
// 128-byte swizzle.
int make_map_out(CUtensorMap* m, void* base, int64_t rows, int64_t blocks, int64_t cols, int64_t F_pad, int64_t ldd,
                 bool box_blocks, bool bf16 = false) {
    EncodeFn enc = encode_fn();
    if (!enc) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const int esz = bf16 ? 2 : 4;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (F_pad * esz) % 16 != 0 || (ldd * esz) % 16 != 0)
        return set_error(FCB_ERR_ARG, "mode product output is not 16-byte aligned");
    cuuint64_t dims[3] = {(cuuint64_t)rows, (cuuint64_t)blocks, (cuuint64_t)cols};
    cuuint64_t strides[2] = {(cuuint64_t)(F_pad * esz), (cuuint64_t)(ldd * esz)};
    cuuint32_t box[3] = {32, box_blocks ? 32u : 1u, box_blocks ? 1u : 32u};
    cuuint32_t estr[3] = {1, 1, 1};
    // 32 elements per line: 128 bytes (FP32) or 64 bytes (BF16), the matching swizzle
    CUresult r = enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     bf16 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return FCB_OK;
}

}  // namespace

// The 2-CTA tile is the default; FCB200_TC_PAIR=0 selects the 1-CTA tile.
static bool use_pair_kernel() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("FCB200_TC_PAIR");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

bool tc_pair_enabled() { return use_pair_kernel(); }

int pad_for(int kind, int64_t n) {
    // TMA needs 16-byte row strides: 8 BF16 or 4 FP32 elements.
    const int64_t q = kind == 1 ? 8 : 4;
    return (int)(((n + q - 1) / q) * q);
}

// Persistent launch of the 2-CTA kernel: one cluster of two per SM pair, capped
// by how many such clusters the device can hold at once (GPCs with an odd SM
// count leave one SM out), so that no cluster waits for another to finish.
template <int KIND, int EPI>
static int launch_pair(fcb200_context* h, int64_t tiles, const CUtensorMap& a_hi, const CUtensorMap& a_lo,
                       const CUtensorMap& b_hi, const CUtensorMap& b_lo, const CUtensorMap& d,
                       const CUtensorMap& dt, const TcParams& p, cudaStream_t s) {
    auto kern = mode_product_tc2_kernel<KIND, EPI>;
    constexpr int SMEM2_BYTES = pair_smem_bytes<EPI>();
    static int max_clusters[64] = {};  // per device, for this kernel
    int& slot = max_clusters[h->device & 63];
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(pair_threads<EPI>(), 1, 1);
    cfg.dynamicSmemBytes = SMEM2_BYTES;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (slot == 0) {
        FCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES));
        cfg.gridDim = dim3(2 * (h->sm_count / 2), 1, 1);
        int n = 0;
        FCB_CUDA(cudaOccupancyMaxActiveClusters(&n, kern, &cfg));
        slot = n > 0 ? n : -1;
    }
    if (slot < 0) return set_error(FCB_ERR_UNSUPPORTED, "mode_product_tc: 2-CTA clusters do not fit");
    const int pairs = (int)(tiles < slot ? tiles : slot);
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    FCB_CUDA(cudaLaunchKernelEx(&cfg, kern, a_hi, a_lo, b_hi, b_lo, d, dt, p));
    return FCB_OK;
}

int mode_product_tc(fcb200_context* h, int kind, const void* A_hi, const void* A_lo, const void* B_hi,
                    const void* B_lo, void* D_hi, void* D_lo, int out_kind, const ModeProduct& mp,
                    cudaStream_t s) {
    if (kind != 1 && kind != 2) return set_error(FCB_ERR_ARG, "mode_product_tc: bad operand kind");
    if (mp.R <= 0 || mp.K <= 0 || mp.M <= 0) return FCB_OK;
    TcParams p;
    p.R = mp.R;
    p.K = mp.K;
    p.M = mp.M;
    p.F = mp.F;
    p.F_pad = mp.F_pad;
    p.ldd = mp.ldd;
    p.sym = mp.sym_full ? 3 : mp.sym_inner ? 2 : mp.sym ? 1 : 0;
    p.inner_upper = mp.inner_upper ? 1 : 0;
    p.packed = mp.packed ? 1 : 0;
    if (mp.packed && !mp.sym_full) return set_error(FCB_ERR_ARG, "mode_product_tc: packed output needs full symmetry");
    p.vec = (mp.F % 8 == 0 && mp.F_pad % 8 == 0 && mp.ldd % 8 == 0) ? 1 : 0;
    p.a_mn = mp.a_mn ? 1 : 0;
    p.b_group = mp.b_group;
    p.b_group_ld = mp.b_group_ld;
    p.Fv = mp.Fv > 0 ? mp.Fv : mp.F;
    p.tma_out = 0;
    if (mp.sym && mp.R != mp.F * mp.M) return set_error(FCB_ERR_ARG, "mode_product_tc: symmetric output needs R = F*M");
    const bool ext = mp.sym_inner || mp.sym_full || mp.a_mn || mp.b_group || p.Fv != mp.F;
    if (ext) {
        // forms of the 2-CTA kernel only; every warp takes the 16-byte store path
        if (!(use_pair_kernel() && h->sm_count >= 2))
            return set_error(FCB_ERR_UNSUPPORTED, "mode_product_tc: grouped / MN-major forms need the 2-CTA tile");
        if (!p.vec || mp.R % 256 != 0 || p.Fv % 8 != 0 || mp.M % 8 != 0)
            return set_error(FCB_ERR_ARG, "mode_product_tc: grouped / MN-major forms need 8-aligned shapes");
        if (mp.sym_inner && (mp.sym || mp.F % 256 != 0 || out_kind != kind))
            return set_error(FCB_ERR_ARG, "mode_product_tc: inner symmetry needs 256-row blocks");
        if (mp.sym_full && (mp.sym || mp.sym_inner || out_kind != 0 || mp.F % 256 != 0 || mp.R != mp.F * mp.M))
            return set_error(FCB_ERR_ARG, "mode_product_tc: full symmetry needs FP32 output, 256-row blocks, R = F*M");
        if (mp.a_mn && (mp.F % 128 != 0 || mp.R % mp.F != 0))
            return set_error(FCB_ERR_ARG, "mode_product_tc: MN-major A needs 128-row blocks");
        if (mp.b_group && mp.b_group % 256 != 0)
            return set_error(FCB_ERR_ARG, "mode_product_tc: B groups must hold whole 256-row tiles");
    }
    p.n_tiles = (int)((mp.M + BN_MAX - 1) / BN_MAX);
    if (h->tune && !mp.sym_inner && !mp.sym_full) {  // autotuned mode-tile count for this shape, if any
        auto it = h->tune->find(tune_key(kind, mp.R, mp.K, mp.M));
        if (it != h->tune->end() && it->second >= p.n_tiles && it->second <= mp.M) p.n_tiles = it->second;
    }
    const int64_t per = (mp.M + p.n_tiles - 1) / p.n_tiles;
    p.bn = (int)(((per + 15) / 16) * 16);
    if ((mp.sym_inner || mp.sym_full) && mp.M > 256) p.bn = 256;  // square 256 × 256 tiles
    p.m_tiles = (int)((mp.R + BM - 1) / BM);
    p.elems_per_row = ROW_BYTES / (kind == 1 ? 2 : 4);
    p.k_chunks = (int)((mp.K + p.elems_per_row - 1) / p.elems_per_row);
    p.out_kind = out_kind;
    p.d_hi = D_hi;
    p.d_lo = D_lo;
    p.status = h->d_status;
    p.wait_ns = h->wait_limit_ns;
    CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
    // B rows: the modes, or (grouped) every group's modes one after another
    const int64_t b_rows = mp.b_group ? mp.b_group_ld * ((mp.R + mp.b_group - 1) / mp.b_group) : mp.M;
    if (mp.a_mn) {
        FCB_TRY(make_map_mn(&ma_hi, A_hi, kind, mp.F, mp.K, mp.R / mp.F, mp.lda, mp.lda_z));
        FCB_TRY(make_map_mn(&ma_lo, A_lo, kind, mp.F, mp.K, mp.R / mp.F, mp.lda, mp.lda_z));
    } else {
        FCB_TRY(make_map(&ma_hi, A_hi, kind, mp.K, mp.R, mp.lda, BM));
        FCB_TRY(make_map(&ma_lo, A_lo, kind, mp.K, mp.R, mp.lda, BM));
    }
    FCB_TRY(make_map(&mb_hi, B_hi, kind, mp.K, b_rows, mp.ldb, p.bn));
    FCB_TRY(make_map(&mb_lo, B_lo, kind, mp.K, b_rows, mp.ldb, p.bn));
    if (use_pair_kernel() && h->sm_count >= 2) {
        // 2-CTA tiles: 256 rows per pair, each CTA loads half of the mode tile
        p.m_tiles = (int)((mp.R + 255) / 256);
        CUtensorMap pb_hi, pb_lo;
        FCB_TRY(make_map(&pb_hi, B_hi, kind, mp.K, b_rows, mp.ldb, p.bn / 2));
        FCB_TRY(make_map(&pb_lo, B_lo, kind, mp.K, b_rows, mp.ldb, p.bn / 2));
        const int64_t tiles2 = (int64_t)p.m_tiles * p.n_tiles;
        // FP32 output with outer symmetry (the third product of the snapshot
        // paths): the epilogue hands whole 32 × 32 blocks to the TMA engine,
        // direct and mirrored, when a warp's 32 rows share one outer index
        CUtensorMap md = ma_hi, mdt = ma_hi;
        p.tma_out = 0;
        if (out_kind == 0 && (mp.sym || mp.sym_full) && p.vec && mp.F % 32 == 0 && mp.R == mp.F * mp.M) {
            FCB_TRY(make_map_out(&md, D_hi, p.Fv, mp.M, mp.M, mp.F_pad, mp.ldd, false));
            FCB_TRY(make_map_out(&mdt, D_hi, p.Fv, mp.M, mp.M, mp.F_pad, mp.ldd, true));
            p.tma_out = 1;
        }
        if (mp.sym_full && p.tma_out != 1)
            return set_error(FCB_ERR_ARG, "mode_product_tc: full symmetry needs the TMA-stored FP32 output");
        // BF16 planes with inner symmetry (the grouped second product): one map
        // per plane, (row in block, block, column), serves the direct box and,
        // with the roles of row and column exchanged, the transposed one.  Its
        // first dimension is F (= Mp), not M: rows p in [M, Mp) are stored too,
        // as the zeros their zero U1c rows give, so that the third product,
        // which reads those padding rows as A rows (and stores none of the K3
        // rows they produce, Fv = M), never reads unwritten memory.  The
        // transposed box, where used, may carry accumulator columns past M
        // (B rows of the next group); they land in padding rows p >= M only.
        if (kind == 1 && out_kind == 1 && mp.sym_inner && p.vec) {
            FCB_TRY(make_map_out(&md, D_hi, mp.F, mp.R / mp.F, mp.M, mp.F_pad, mp.ldd, false, true));
            FCB_TRY(make_map_out(&mdt, D_lo, mp.F, mp.R / mp.F, mp.M, mp.F_pad, mp.ldd, false, true));
            p.tma_out = 2;
        }
        // the grouped second product (K of a few hundred) is bound by its
        // epilogue: twice the epilogue warps
        if (p.sym == 2) {
            if (kind == 1) return launch_pair<1, 8>(h, tiles2, ma_hi, ma_lo, pb_hi, pb_lo, md, mdt, p, s);
            return launch_pair<2, 8>(h, tiles2, ma_hi, ma_lo, pb_hi, pb_lo, md, mdt, p, s);
        }
        if (kind == 1) return launch_pair<1, 4>(h, tiles2, ma_hi, ma_lo, pb_hi, pb_lo, md, mdt, p, s);
        return launch_pair<2, 4>(h, tiles2, ma_hi, ma_lo, pb_hi, pb_lo, md, mdt, p, s);
    }
    const int64_t tiles = (int64_t)p.m_tiles * p.n_tiles;
    const int grid = (int)(tiles < h->sm_count ? tiles : h->sm_count);
    // The shared-memory limit is a per-device attribute of the function: set
    // it on every launch (a handle per device may share this process).
    if (kind == 1) {
        FCB_CUDA(cudaFuncSetAttribute(mode_product_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      SMEM_BYTES));
        mode_product_tc_kernel<1><<<grid, NUM_THREADS, SMEM_BYTES, s>>>(ma_hi, ma_lo, mb_hi, mb_lo, p);
    } else {
        FCB_CUDA(cudaFuncSetAttribute(mode_product_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      SMEM_BYTES));
        mode_product_tc_kernel<2><<<grid, NUM_THREADS, SMEM_BYTES, s>>>(ma_hi, ma_lo, mb_hi, mb_lo, p);
    }
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
