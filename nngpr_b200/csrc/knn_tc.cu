// Exact k-nearest-neighbour search with a tensor-core (tcgen05) screen, B200 (sm_100a).
//
// Same contract and results as the screened SIMT kernel in knn.cu (exact lists: the FP32
// distance of the CPU restatement, ascending, lower index first on ties, -1 padding, ref cut).
// What changes is who computes the screening scores s_qr = |rc|^2 - 2 qc.rc (centred
// coordinates, the candidate test being s < tau - |qc|^2 + eps) and how candidates are merged:
//
//   * the scores of a 128-query x 128-ref tile are one UMMA product D = A B^T in TMEM
//     (tcgen05.mma kind::tf32, M=128, N=128, FP32 accumulate).  To keep FP32-level accuracy each
//     operand a = a_hi + a_lo is split (a_hi = a rounded to TF32, a_lo = a - a_hi, exact), and
//     A' = [a_hi | a_hi | a_lo], B' = [b_hi | b_lo | b_hi] (each block d+1 wide: the d centred
//     coordinates, the constant 1 and the |rc|^2 column) so that A' B'^T = a_hi b_hi + a_hi b_lo + a_lo b_hi.
//     The dropped and truncated terms are below 2^-21 |a||b| per product, the FP32 accumulation
//     adds at most K' ulps; eps = 2^-16 (|qc| + max|rc|)^2 covers both with a margin of 4 or more,
//     so every ref the exact algorithm inserts still passes the screen;
//   * persistent CTAs (work items = query tiles handed out heaviest first through a global
//     counter), 160 threads: warp 4 allocates TMEM (two 128-column accumulators, or one when
//     three CTAs share the SM) and
//     one of its lanes issues the TMA bulk copies of ref tiles into a shared-memory ring (operands
//     and exact coordinates in one copy) and the MMAs; warps 0-3 are the epilogue, warp w owning
//     query rows 32w..32w+31 (its TMEM lane quadrant).  Up to three CTAs share an SM when shared
//     memory allows (small d): the epilogue is latency-bound, and every extra warp per scheduler
//     shows (d = 3: 30.8 ms with two CTAs per SM, 23.1 ms with three, n = 434,874).  For d = 12
//     and 16, where one CTA fills an SM, a work item is two query tiles: both MMA chains read the
//     same staged ref tile and 8 epilogue warps share the SM (d = 16, n = 1M: 235 -> 173 ms);
//   * epilogue: each 32-column chunk of a row is one tcgen05.ld (issued one chunk ahead into a
//     second register set), screened with three-input min over groups of 8 columns against the
//     row's threshold into a candidate mask (skipped when no row of the warp has one); the
//     accumulator buffer is freed as soon as the tile's four chunks are read.  Then each lane
//     walks the candidates of its row in the whole tile, one per warp iteration (so one
//     iteration serves every row that has a candidate), and rescores them exactly (exact
//     coordinates from the same smem stage, the oracle's arithmetic); survivors of the row's
//     current bound are compacted with ballots into a
//     per-warp queue.  Once 32 entries are queued the warp drains them into the rows' lists: each
//     row keeps its best m as a max-heap of 64-bit keys (distance bits << 32 | index) in shared
//     memory, 32 entries go in per pass, one per lane, entries of one row serialised by match_any.
//     The key order is (distance, index), so the final sets do not depend on insertion order; at
//     the end of a work item each heap is sorted across the warp (bitonic) and written out;
//   * mbarriers: b_full (TMA -> MMA), b_empty (MMA commit + 4 epilogue warps -> producer),
//     t_full (MMA commit -> epilogue), t_empty (4 epilogue warps -> MMA), a_ready (query operand
//     written by the epilogue -> MMA).  Every wait is bounded; on a timeout the CTA raises
//     NNGP_FLAG_TIMEOUT, drains what it issued (bounded), frees TMEM and returns.
// No TMA multicast and no cluster launch.
#include <algorithm>
#include <string>
#include <type_traits>

#include "common.cuh"
#include "knn_tc.cuh"

namespace nngp {
namespace tc {

constexpr int QT = kTcQueryTile;  // queries per tile (UMMA M)
constexpr int RT = kTcRefTile;    // refs per tile (UMMA N)
static_assert(RT == 128, "the epilogue screens a ref tile as four 32-column chunks");
constexpr int THREADS = 5 * 32;   // layout self-test: 4 epilogue warps + the MMA warp
constexpr int LIST = 32;       // largest num_nn
constexpr int HS = 33;         // heap row stride in 64-bit keys (odd: rows of a warp hit distinct banks)
constexpr int DRAIN_AT = 32;   // queued entries that trigger a drain at the end of a tile (8: +2%, 128: +7% at d = 3)
constexpr int QCAP = 64;       // key queue entries per epilogue warp (a drain runs before a batch
                               // that could overflow it)
constexpr int CQCAP = 96;      // screened candidates queued per epilogue warp for rescoring
constexpr int MAX_STAGES = 8;  // ring stages (mbarrier slots)
constexpr uint32_t kSelftestCols = 2 * RT;  // TMEM columns of the layout self-test
constexpr float kEpsTc = 1.52587890625e-05f;       // 2^-16: TF32 x3 split
constexpr float kEpsBf = 6.103515625e-05f;         // 2^-14: BF16 x3 split
constexpr float kPadNorm = 1.7014118346046923e38f;  // 2^127: padded refs never pass a finite screen
// list key: FP32 distance bits (non-negative, so integer order = float order) << 32 | index;
// an empty slot is (+inf, 0xffffffff), larger than every real entry, read back as index -1
constexpr uint64_t kEmptyKey = (uint64_t)0x7F800000u << 32 | 0xFFFFFFFFu;

// D: padded dimension; QTILES: 128-query tiles per work item (their MMAs share each staged ref
// tile; 4 epilogue warps per query tile, one per TMEM lane quadrant).
// Operands: D <= 8 a TF32 x3 split (kind::tf32, K = 8 per MMA, 4-byte elements); D >= 12 a BF16 x3
// split (kind::f16, K = 16 per MMA, 2-byte elements): half the bytes per ref tile and, at the
// tensor pipe's doubled BF16 rate, 4 instead of 7 MMA steps per tile at D = 16.
template <int D, int QTILES>
struct Cfg {
    static constexpr bool BF16 = D >= 12;
    static constexpr int ESZ = BF16 ? 2 : 4;        // operand element bytes
    static constexpr int EPC = 16 / ESZ;            // elements per 16-byte core-matrix row
    static constexpr int KMMA = BF16 ? 16 : 8;      // UMMA K of one instruction
    static constexpr float EPS = BF16 ? kEpsBf : kEpsTc;
    static constexpr int EPI_WARPS = 4 * QTILES;
    static constexpr int ROWS = QT * QTILES;        // queries per work item
    static constexpr int U = D + 1;                 // coordinates + the norm column
    static constexpr int KP = (3 * U + KMMA - 1) / KMMA * KMMA;  // split operand width
    static constexpr int NMMA = KP / KMMA;
    // operand rows of exactly 128 bytes (d = 16, 20 BF16, d = 8 TF32) use the 128-byte swizzle:
    // operands 1024-byte aligned, one MMA's K slice = 32 bytes further along the row
    static constexpr bool SW128 = KP * ESZ == 128;
    static constexpr int ALIGN = SW128 ? 1024 : 128;
    static constexpr int DP = (D + 3) / 4 * 4;      // exact-coordinate row length
    static constexpr int OP_BYTES = RT * KP * ESZ;  // B operand block of a ref tile
    static constexpr int EX_BYTES = RT * DP * 4;    // exact coordinates of a ref tile
    // where a tile record keeps its refs' point indices: the spare last slot of each exact-coordinate
    // row when DP > D (1), a block after the coordinates for the BF16 shapes (2); D = 4 and 8 read
    // them from ref_perm (0)
    static constexpr int IX_MODE = DP > D ? 1 : (BF16 ? 2 : 0);
    static constexpr int IX_BYTES = IX_MODE == 2 ? RT * 4 : 0;
    // a ref tile in global memory: [B operand | exact coordinates | indices]; only the B operand
    // is staged in shared memory (the MMAs' input), so a stage is free again as soon as its MMAs
    // complete.  The screen passes about one pair in 3,000 at d = 16: the epilogue reads those
    // pairs' exact coordinates and indices from the record in global memory, 32 at a time.
    static constexpr int TILE_BYTES = OP_BYTES + EX_BYTES + IX_BYTES;
    // d = 16: a stage holds two ref tiles, multiplied by one MMA of N = 256 per query tile and K
    // slice (half the MMA instructions and 12 KB of operand reads per 256 x 128 x 16 instead of
    // 16 KB); its accumulators fill the 512 TMEM columns, single-buffered
    static constexpr bool PAIR = D == 16 && QTILES == 2;
    static constexpr int TPS = PAIR ? 2 : 1;        // ref tiles per stage
    static constexpr int RS = RT * TPS;             // refs per stage (MMA N)
    static constexpr int STAGE_BYTES = OP_BYTES * TPS;
    static constexpr int A_TILE = QT * KP * ESZ;    // query operand of one query tile
    static constexpr int A_BYTES = A_TILE * QTILES;
    static constexpr int LIST_BYTES = ROWS * HS * 8;  // one heap of keys per query
    static constexpr int QUEUE_BYTES = EPI_WARPS * QCAP * (8 + 1);  // key + row
    static constexpr int CQ_BYTES = EPI_WARPS * CQCAP * 8;          // ref position << 5 | row
    static constexpr int BAR_BYTES = 256;
    static constexpr int FIXED = ALIGN + A_BYTES + LIST_BYTES + QUEUE_BYTES + CQ_BYTES + BAR_BYTES;  // ALIGN: base slack
    // as many CTAs per SM (up to 3) as hold at least 2 stages each: more epilogue warps per
    // scheduler.  Three CTAs share TMEM with one accumulator buffer each (the epilogue frees it
    // as soon as a tile's scores are in registers); one or two CTAs double-buffer it.
    static constexpr int ST3 = (75 * 1024 - FIXED) / STAGE_BYTES;
    static constexpr int ST2 = (112 * 1024 - FIXED) / STAGE_BYTES;
    static constexpr int ST1 = (220 * 1024 - FIXED) / STAGE_BYTES;
    static constexpr int CTAS_PER_SM = ST3 >= 2 ? 3 : (ST2 >= 2 ? 2 : 1);
    static constexpr int STN = CTAS_PER_SM == 3 ? ST3 : (CTAS_PER_SM == 2 ? ST2 : ST1);
    static constexpr int STAGES = STN > MAX_STAGES ? MAX_STAGES : STN;
    // A CTA alone on its SM streams its tiles from a warp of its own: the MMA warp then waits
    // only for a staged tile and a free accumulator buffer, never for a stage to be refilled,
    // and each copy starts as soon as the MMAs of the stage's previous tile complete.  With 2 or
    // 3 CTAs per SM the other CTAs fill those gaps, and the register budget has no room for
    // another warp: the MMA warp issues the copies itself.
    static constexpr bool TMA_WARP = CTAS_PER_SM == 1;
    static constexpr int THREADS = (EPI_WARPS + 1 + (TMA_WARP ? 1 : 0)) * 32;
    static constexpr int SMEM = FIXED + STAGES * STAGE_BYTES;
    static constexpr int NBUF = (CTAS_PER_SM == 3 || PAIR) ? 1 : 2;  // accumulator buffers in TMEM
    static constexpr uint32_t BUF_COLS = RS * QTILES;                 // one buffer: a stage per query tile
    static constexpr uint32_t TMEM_COLS = NBUF * BUF_COLS;  // a power of two >= 32, <= 512
    static_assert(TMEM_COLS <= 512 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "TMEM columns");
    static_assert(CTAS_PER_SM * TMEM_COLS <= 512, "TMEM of the CTAs sharing an SM");
    static_assert(STAGES >= 2, "ref tile too large for two stages");
};

// byte offset of element (row, k) of a K-major UMMA operand with `rows` rows and ESZ-byte
// elements.  SW = false: no swizzle, core matrices of 8 rows x 16 bytes.  SW = true: the 128-byte
// swizzle for rows of exactly 128 bytes (K * ESZ = 128): 8-row atoms of 1 KB, row r of an atom at
// byte 128 (r % 8), its 16-byte chunk c at chunk c ^ (r % 8) -- the order in which the tensor core
// reads a 1024-byte-aligned atom with SWIZZLE_128B (bank-conflict free, unlike the no-swizzle
// layout whose 8 rows of one core matrix share 128 bytes)
template <int ESZ = 4, bool SW = false>
__host__ __device__ __forceinline__ uint32_t op_offset(int row, int k, int rows) {
    if constexpr (SW) {
        const uint32_t byte = (uint32_t)k * ESZ;
        return (uint32_t)(row >> 3) * 1024u + (uint32_t)(row & 7) * 128u +
               ((((byte >> 4) ^ (uint32_t)(row & 7)) & 7u) << 4) + (byte & 15u);
    } else {
        constexpr int EPC = 16 / ESZ;
        return (uint32_t)((k / EPC) * (rows / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k % EPC) * ESZ);
    }
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x rounded to the nearest BF16 (ties to even), as its 16-bit pattern and as a float
__device__ __forceinline__ uint16_t bf16_bits(float x) {
    uint16_t r;
    asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float bf16_value(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Element k of one row of a split operand: blocks [hi | hi | lo] (query side, lo_block = 2) or
// [hi | lo | hi] (ref side, lo_block = 1) of the U values v, then zeros; the products
// A' B'^T = a_hi b_hi + a_hi b_lo + a_lo b_hi.  Stored at `dst` as TF32 (float) or BF16.
template <bool BF16, int U, bool SW = false>
__device__ __forceinline__ void put_split(unsigned char *dst_row_base, int row, int rows, int k, int lo_block,
                                          const float (&v)[U]) {
    float val = 0.f;
    const int blk = k / U, f = k - blk * U;
    if constexpr (BF16) {
        uint16_t bits = 0;
        if (blk < 3) {
            const uint16_t hi = bf16_bits(v[f]);
            bits = (blk == lo_block) ? bf16_bits(v[f] - bf16_value(hi)) : hi;
        }
        *reinterpret_cast<uint16_t *>(dst_row_base + op_offset<2, SW>(row, k, rows)) = bits;
    } else {
        if (blk < 3) {
            const float hi = tf32_round(v[f]);
            val = (blk == lo_block) ? (v[f] - hi) : hi;
        }
        *reinterpret_cast<float *>(dst_row_base + op_offset<4, SW>(row, k, rows)) = val;
    }
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, bool sw128 = false) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    if (sw128) d |= (uint64_t)2 << 61;  // layout SWIZZLE_128B (else 0, SWIZZLE_NONE); base offset 0, lbo mode 0
    return d;
}

// Descriptor of K slice i (K = KMMA elements) of a K-major operand at smem address base with
// `rows` rows: no swizzle (LBO between 16-byte K chunks = rows / 8 core matrices, SBO 128 between
// 8-row groups; one slice spans two chunks) or the 128-byte swizzle (rows of 128 bytes, 8-row atoms
// of 1 KB = SBO, LBO unused (16), the slice starting 32 bytes further along the row)
template <bool SW, int ESZ, int KMMA>
__device__ __forceinline__ uint64_t op_desc(uint32_t base, int rows, int i) {
    if constexpr (SW) return smem_desc(base + (uint32_t)(i * KMMA * ESZ), 16, 1024, true);
    else return smem_desc(base + (uint32_t)(i * 2 * (rows / 8) * 128), (uint32_t)((rows / 8) * 128), 128);
}

// instruction descriptors: F32 accumulate, both operands K-major, N = RT, M = QT; A and B TF32
// (kind::tf32, format 2) or BF16 (kind::f16, format 1) -- A and B of one type
constexpr uint32_t kIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(RT >> 3) << 17) | ((uint32_t)(QT >> 4) << 24);
constexpr uint32_t kIdescBf16 =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(RT >> 3) << 17) | ((uint32_t)(QT >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate,
                                         uint32_t idesc = kIdesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate,
                                         uint32_t idesc = kIdescBf16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// instruction descriptor of an M = QT, N = n product (F32 accumulate, K-major A and B)
constexpr uint32_t idesc_of(bool bf16, int n) {
    return (1u << 4) | ((bf16 ? 1u : 2u) << 7) | ((bf16 ? 1u : 2u) << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(QT >> 4) << 24);
}

template <bool BF16, int N = RT>
__device__ __forceinline__ void mma_op(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    if constexpr (BF16) mma_bf16(tmem_d, adesc, bdesc, accumulate, idesc_of(true, N));
    else mma_tf32(tmem_d, adesc, bdesc, accumulate, idesc_of(false, N));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 columns of this thread's TMEM lane, no wait (the caller issues tcgen05.wait::ld)
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// Wait for this thread's outstanding tcgen05.ld; the registers of the load are operands, so no
// use of them can be scheduled before the wait.
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// Max-heap of the m best keys (root = current m-th best): replace the root by x when x is
// smaller and sift it down.
__device__ __forceinline__ void heap_insert(uint64_t *h, int m, uint64_t x) {
    if (!(x < h[0])) return;
    int i = 0;
    while (true) {
        int c = 2 * i + 1;
        if (c >= m) break;
        uint64_t kc = h[c];
        if (c + 1 < m) {
            const uint64_t k2 = h[c + 1];
            if (k2 > kc) {
                kc = k2;
                ++c;
            }
        }
        if (kc <= x) break;
        h[i] = kc;
        i = c;
    }
    h[i] = x;
}

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Ref tiles in global memory: per tile [B' operand block (UMMA layout) | exact coordinates (RT x DP)
// | point indices (RT int32, -1 for padding)].  xs: scaled refs (n_pad x DP, zero padded); acc:
// per-feature sums for the centre.
template <int D>
__global__ void build_tc_tiles_kernel(const float *__restrict__ xs, int64_t n, int64_t n_pad,
                                      const double *__restrict__ acc, const int32_t *__restrict__ perm,
                                      unsigned char *__restrict__ tiles, unsigned int *__restrict__ r2max_bits) {
    using C = Cfg<D, 1>;  // the ref-tile layout does not depend on the query tiles
    float c[D];
#pragma unroll
    for (int f = 0; f < D; ++f) c[f] = n > 0 ? (float)(acc[f] / (double)n) : 0.f;
    float mx = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pad; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / RT;
        const int row = (int)(i - t * RT);
        unsigned char *base = tiles + t * C::TILE_BYTES;
        float b[C::U];
        float ex[C::DP];
#pragma unroll
        for (int k = 0; k < C::DP; ++k) ex[k] = 0.f;
        if (i < n) {
            float nr = 0.f;
#pragma unroll
            for (int f = 0; f < D; ++f) {
                const float r = xs[(perm ? (int64_t)perm[i] : i) * C::DP + f];
                const float rc = r - c[f];
                ex[f] = r;
                b[f] = -2.f * rc;
                nr = fmaf(rc, rc, nr);
            }
            b[D] = nr;
            mx = fmaxf(mx, nr);
        } else {
#pragma unroll
            for (int f = 0; f < D; ++f) b[f] = 0.f;
            b[D] = kPadNorm;
        }
        for (int k = 0; k < C::KP; ++k) put_split<C::BF16, C::U, C::SW128>(base, row, RT, k, 1, b);  // [b_hi | b_lo | b_hi]
        const int32_t pidx = i < n ? (int32_t)(perm ? (int64_t)perm[i] : i) : -1;
        if (C::IX_MODE == 1) ex[C::DP - 1] = __int_as_float(pidx);
        float *exo = reinterpret_cast<float *>(base + C::OP_BYTES) + row * C::DP;
#pragma unroll
        for (int k = 0; k < C::DP; ++k) exo[k] = ex[k];
        if (C::IX_MODE == 2) reinterpret_cast<int32_t *>(base + C::OP_BYTES + C::EX_BYTES)[row] = pidx;
    }
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    if ((threadIdx.x & 31) == 0) atomicMax(r2max_bits, __float_as_uint(mx));
}

template <int D, int QTILES>
__global__ void __launch_bounds__(Cfg<D, QTILES>::THREADS, Cfg<D, QTILES>::CTAS_PER_SM)
    knn_tc_kernel(const unsigned char *__restrict__ tiles_g,
                                                         const float *__restrict__ qs,
                                                         const double *__restrict__ acc,
                                                         const unsigned int *__restrict__ r2max_bits,
                                                         const float *__restrict__ seeds,
                                                         const int32_t *__restrict__ rows_perm,
                                                         const int32_t *__restrict__ row_off,
                                                         const int64_t *__restrict__ dev_sizes,
                                                         const TcItems items,
                                                         const int32_t *__restrict__ ref_perm,
                                                         const int32_t *__restrict__ tile_off,
                                                         const int32_t *__restrict__ tile_list,
                                                         int *__restrict__ work_counter, int64_t n_query,
                                                         int64_t n_ref, int has_cut, int64_t cut, int m,
                                                         int64_t out_base, int32_t *__restrict__ out,
                                                         int32_t *__restrict__ flags, uint64_t wait_ns) {
    using C = Cfg<D, QTILES>;
    constexpr int S = C::STAGES;
    constexpr int EPI_WARPS = C::EPI_WARPS;
    constexpr unsigned FULL = 0xffffffffu;
    // base aligned to C::ALIGN: 1024 for the swizzled operands (their atoms), else 128 (the
    // no-swizzle operands and the bulk copies need 16)
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + (C::ALIGN - 1)) & ~uintptr_t(C::ALIGN - 1));
    unsigned char *sA = sm;
    unsigned char *sB = sA + C::A_BYTES;
    uint64_t *H = reinterpret_cast<uint64_t *>(sB + S * C::STAGE_BYTES);  // [ROWS][HS] heaps
    unsigned char *qbase = reinterpret_cast<unsigned char *>(H + C::ROWS * HS);
    uint64_t *cqbase = reinterpret_cast<uint64_t *>(qbase + C::QUEUE_BYTES);  // [EPI_WARPS][CQCAP] candidates
    uint64_t *bars = cqbase + EPI_WARPS * CQCAP;
    uint64_t *b_full = bars;                    // [S <= MAX_STAGES]
    uint64_t *b_empty = bars + MAX_STAGES;      // [S <= MAX_STAGES]
    uint64_t *t_full = bars + 2 * MAX_STAGES;   // [2]
    uint64_t *t_empty = t_full + 2;             // [2]
    uint64_t *a_ready = t_full + 4;             // [1]
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(t_full + 5);
    volatile int *s_item = reinterpret_cast<volatile int *>(t_full + 6);
    volatile int *s_abort = reinterpret_cast<volatile int *>(t_full + 7);
    static_assert((2 * MAX_STAGES + 8) * 8 <= C::BAR_BYTES, "barrier block");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer_warp = warp == EPI_WARPS;                 // MMA issue (and the copies without TMA_WARP)
    const bool copy_warp = C::TMA_WARP && warp == EPI_WARPS + 1;  // the copies with TMA_WARP
    // Rows: positions [first_row, first_row + n_rows) of rows_perm (point indices; the positions
    // themselves when rows_perm is null), from dev_sizes = {first_row, n_rows, n_items} on the
    // device or {0, n_query, ceil(n_query / ROWS)}; work item g is positions
    // [row_off[g], row_off[g + 1]) (at most ROWS) or ROWS consecutive positions.  Refs: with
    // tile_list (pruned search), group g streams the tiles tile_list[tile_off[g] .. tile_off[g + 1])
    // of tiles_g (each staged tile carries its refs' point indices; ref_perm is the same map in
    // global memory, kept for the host's bookkeeping), and j < limit(i) is checked per
    // candidate; otherwise refs in index order up to the largest limit of the group's rows (the
    // rows of a group ascend).  Items: see TcItems.
    const bool pruned = tile_list != nullptr;
    const int64_t first_row = dev_sizes ? dev_sizes[0] : 0;
    const int64_t n_rows = dev_sizes ? dev_sizes[1] : n_query;
    const int64_t n_items = dev_sizes ? dev_sizes[2] : (n_query + C::ROWS - 1) / C::ROWS;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);  // the MMA commit: the epilogue never reads a stage
        }
        // accumulator barriers: one pair per TMEM buffer, or with PAIR one pair per query tile (its
        // 256 columns are released by its own four warps, so the MMAs of one query tile's next
        // stage overlap the other tile's epilogue)
        for (int b = 0; b < (C::PAIR ? QTILES : C::NBUF); ++b) {
            mbar_init(&t_full[b], 1);
            mbar_init(&t_empty[b], C::PAIR ? 4 : EPI_WARPS);
        }
        mbar_init(a_ready, EPI_WARPS * 32);
        *s_abort = 0;
        fence_mbar_init();
    }
    if (producer_warp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(const_cast<uint32_t *>(tmem_slot))),
                     "r"(C::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const float rmax = sqrtf(__uint_as_float(*r2max_bits)) * 1.0001f;

    uint32_t g_tile = 0;  // stages this CTA has streamed (phases of the ring and TMEM buffers)
    uint32_t it = 0;      // work items this CTA has processed (phase of a_ready)
    bool aborted = false;
    uint32_t tma_issued = 0, tma_landed = 0;  // producer lane: copies issued / waited for (drain on abort)
    int last_tf = -1;                         // producer lane: accumulator barrier of the last commit
    uint32_t last_tf_par = 0;                 // and the parity of that phase

    auto limit_of = [&](int64_t qq) -> int64_t {
        if (!has_cut) return n_ref;
        int64_t l = qq + cut;
        return l < 0 ? 0 : (l > n_ref ? n_ref : l);
    };

    while (true) {
        if (threadIdx.x == 0) *s_item = atomicAdd(work_counter, 1);
        __syncthreads();
        const int item = *s_item;
        const bool stop = (item >= n_items) || (*s_abort != 0);
        __syncthreads();
        if (stop) break;
        const int64_t desc = items.order ? (int64_t)items.order[item] : -1;  // the item's descriptor
        const int64_t qtile = desc >= 0 ? (int64_t)items.group[desc] : (has_cut ? (n_items - 1 - item) : item);
        const int32_t out_slot = desc >= 0 ? items.slot[desc] : -1;  // >= 0: partial lists for a merge
        int64_t q0, n_item_rows;  // the item's first row position and its row count
        if (row_off) {
            q0 = row_off[qtile];
            n_item_rows = row_off[qtile + 1] - q0;
        } else {
            q0 = first_row + qtile * C::ROWS;
            n_item_rows = min((int64_t)C::ROWS, first_row + n_rows - q0);
        }
        auto point_of = [&](int64_t pos) -> int64_t { return rows_perm ? (int64_t)rows_perm[pos] : pos; };
        uint32_t tfirst = 0, ntiles;  // the item's tiles: positions [tfirst, tfirst + ntiles) of the group's range
        if (desc >= 0) {
            tfirst = (uint32_t)items.t0[desc];
            ntiles = (uint32_t)(items.t1[desc] - items.t0[desc]);
        } else if (pruned) {
            ntiles = (uint32_t)(tile_off[qtile + 1] - tile_off[qtile]);
        } else {
            const int64_t block_limit = limit_of(point_of(q0 + n_item_rows - 1));
            ntiles = (uint32_t)((block_limit + RT - 1) / RT);
        }
        const int32_t *tl = pruned ? tile_list + tile_off[qtile] + tfirst : nullptr;  // this item's ref tiles
        // the item's stages: its tiles one per stage, or two (PAIR: tiles 2u and 2u + 1 in stage u,
        // the second half of the last stage empty when ntiles is odd)
        const uint32_t nstg = (ntiles + C::TPS - 1) / C::TPS;
        const uint32_t G = g_tile;  // stages this CTA streamed before the item
        // stage buffer g % S is free once the MMAs of stage g - S are done with it
        auto wait_empty = [&](uint32_t g) -> bool {
            const uint32_t k = g / S;
            return mbar_wait_bounded(&b_empty[g % S], (k & 1) ^ 1, wait_ns);
        };
        // the tile record the item's t-th tile comes from
        auto tile_at = [&](uint32_t t) -> int64_t { return pruned ? (int64_t)tl[t] : (int64_t)(tfirst + t); };
        // stage g: the B operand of tile record ta, and of tb after it when tb >= 0
        auto issue_stage = [&](uint32_t g, int64_t ta, int64_t tb) {
            const uint32_t s = g % S;
            mbar_arrive_expect_tx(&b_full[s], (uint32_t)C::OP_BYTES * (tb >= 0 ? 2u : 1u));
            tma_bulk_g2s(sB + s * C::STAGE_BYTES, tiles_g + ta * C::TILE_BYTES, C::OP_BYTES, &b_full[s]);
            if (tb >= 0)
                tma_bulk_g2s(sB + s * C::STAGE_BYTES + C::OP_BYTES, tiles_g + tb * C::TILE_BYTES, C::OP_BYTES,
                             &b_full[s]);
            tma_issued = g + 1;
        };
        auto issue_tma = [&](uint32_t g, int64_t t) { issue_stage(g, t, -1); };

        if (copy_warp) {
            // the item's tiles in order, each as soon as its stage is free (no query operand
            // needed); the warp reads the tile list 32 entries at a time, so no dependent global
            // load sits between two copies
            int64_t ent = 0;
            for (uint32_t u = 0; u < nstg; ++u) {
                const uint32_t t = u * C::TPS;  // the stage's first tile (t + 1 is in the same batch of 32)
                if ((t & 31u) == 0) ent = t + lane < ntiles ? tile_at(t + lane) : 0;
                const int64_t cur = __shfl_sync(FULL, ent, (int)(t & 31u));
                const int64_t cur2 = C::PAIR ? __shfl_sync(FULL, ent, (int)((t + 1) & 31u)) : 0;
                bool ok = true;
                if (lane == 0) {
                    ok = wait_empty(G + u);
                    if (ok) issue_stage(G + u, cur, (C::PAIR && t + 1 < ntiles) ? cur2 : (int64_t)-1);
                }
                if (!__shfl_sync(FULL, ok, 0)) {
                    aborted = true;
                    break;
                }
            }
            __syncwarp();
        } else if (producer_warp) {
            if (lane == 0) {
                if (!mbar_wait_bounded(a_ready, it & 1, wait_ns)) aborted = true;  // query operand of this item
                if constexpr (!C::TMA_WARP) {
                    for (uint32_t k = 0; k < (uint32_t)S && k < ntiles && !aborted; ++k) {
                        if (!wait_empty(G + k)) {
                            aborted = true;
                            break;
                        }
                        issue_tma(G + k, tile_at(k));
                    }
                }
                // list entry of the next refill, read one refill ahead
                int64_t next_fill = (!C::TMA_WARP && (uint32_t)S < ntiles) ? tile_at(S) : 0;
                const uint32_t a_addr = smem_addr(sA);
                for (uint32_t t = 0; t < nstg && !aborted; ++t) {  // t: the item's stage
                    const uint32_t g = G + t;
                    const uint32_t s = g % S, b = g % C::NBUF, use = g / C::NBUF;
                    if (!mbar_wait_bounded(&b_full[s], (g / S) & 1, wait_ns)) {
                        aborted = true;
                        break;
                    }
                    tma_landed = g + 1;
                    const uint32_t b_addr = smem_addr(sB + s * C::STAGE_BYTES);
                    bool stop_mma = false;
#pragma unroll
                    for (int qt = 0; qt < QTILES; ++qt) {  // every query tile against the same staged refs
                        if (C::PAIR || qt == 0) {  // the accumulator(s) this query tile writes are free
                            const uint32_t tb = C::PAIR ? (uint32_t)qt : b;
                            if (!mbar_wait_bounded(&t_empty[tb], ((C::PAIR ? g : use) & 1) ^ 1, wait_ns)) {
                                stop_mma = true;
                                break;
                            }
                            tc_fence_after();
                        }
                        const uint32_t d_tmem = tmem_base + b * C::BUF_COLS + qt * C::RS;
                        const uint32_t aq = a_addr + qt * C::A_TILE;
#pragma unroll
                        for (int i = 0; i < C::NMMA; ++i) {  // one K slice per MMA
                            const uint64_t ad = op_desc<C::SW128, C::ESZ, C::KMMA>(aq, QT, i);
                            const uint64_t bd = op_desc<C::SW128, C::ESZ, C::KMMA>(b_addr, C::RS, i);
                            mma_op<C::BF16, C::RS>(d_tmem, ad, bd, i > 0 ? 1u : 0u);
                        }
                        if (C::PAIR) {
                            mma_commit(&t_full[qt]);
                            last_tf = qt;
                            last_tf_par = g & 1;
                        }
                    }
                    if (stop_mma) {
                        aborted = true;
                        break;
                    }
                    if (!C::PAIR) {
                        mma_commit(&t_full[b]);
                        last_tf = (int)b;
                        last_tf_par = use & 1;
                    }
                    mma_commit(&b_empty[s]);
                    if constexpr (!C::TMA_WARP) {
                        const uint32_t gr = g - 1 + S;  // refill the stage that MMA g-1 used
                        if (t > 0 && gr < G + nstg) {
                            const int64_t cur = next_fill;
                            if (gr + 1 < G + nstg) next_fill = tile_at(gr + 1 - G);
                            if (!wait_empty(gr)) {
                                aborted = true;
                                break;
                            }
                            issue_tma(gr, cur);
                        }
                    }
                }
            }
            __syncwarp();
        } else {
            // ---------------- epilogue warps ----------------
            // warp w serves query tile w / 4 through TMEM lane quadrant w % 4 (a warp reaches the
            // lanes of its own quadrant only)
            const int qtw = warp >> 2, quad = warp & 3;
            // query row in the work item.  PAIR: the rows are dealt out to the warps in turn (row r
            // to warp r mod EPI_WARPS), so that the candidates of a spatially clustered run of rows
            // spread over the warps that must release an accumulator together (-1 % at d = 16; the
            // other shapes keep runs of 32)
            const int row = C::PAIR ? lane * EPI_WARPS + warp : warp * 32 + lane;
            const bool active = row < n_item_rows;
            const int64_t q = active ? point_of(q0 + row) : 0;  // the point's index
            const int64_t limit = active ? limit_of(q) : 0;
            float qo[D], qc[D];
            float nq = 0.f;
#pragma unroll
            for (int f = 0; f < D; ++f) {
                qo[f] = active ? qs[q * C::DP + f] : 0.f;
                const float cf = n_ref > 0 ? (float)(acc[f] / (double)n_ref) : 0.f;
                qc[f] = qo[f] - cf;
                nq = fmaf(qc[f], qc[f], nq);
            }
            const float span = sqrtf(nq) * 1.0001f + rmax;
            const float eps = C::EPS * span * span;
            {  // query operand row: A' = [a_hi | a_hi | a_lo], a = [qc, 1]
                float a[C::U];
#pragma unroll
                for (int f = 0; f < D; ++f) a[f] = active ? qc[f] : 0.f;
                a[D] = active ? 1.f : 0.f;
                for (int k = 0; k < C::KP; ++k)
                    put_split<C::BF16, C::U, C::SW128>(sA + qtw * C::A_TILE, quad * 32 + lane, QT, k, 2, a);
            }
            fence_proxy_async_smem();
            mbar_arrive(a_ready);

            // this warp's rows: row rr's heap at heap[rr * HS .. + m)
            uint64_t *heap = H + (warp * 32) * HS;
            for (int rr = 0; rr < 32; ++rr) heap[rr * HS + lane] = kEmptyKey;
            uint64_t *qk = reinterpret_cast<uint64_t *>(qbase) + warp * QCAP;  // queued keys
            uint8_t *qr = qbase + EPI_WARPS * QCAP * 8 + warp * QCAP;           // their rows
            __syncwarp();
            // rows past the last query never take candidates
            const float tq_off = active ? pos_inf<float>() : neg_inf<float>();
            // a proven upper bound of the row's m-th distance (seeded prefix search), else +inf
            const float seed_r = (active && seeds) ? seeds[q] : pos_inf<float>();
            float worst = seed_r;  // min(seed, distance of the heap root = m-th best so far)
            float tq = fminf((worst - nq) + eps, tq_off);  // screening threshold of this row
            int qcount = 0;
            // insert the queued entries: 32 at a time, each lane into its entry's row heap; entries
            // of one row go in one after the other (match_any groups), so any order gives the same heap set
            auto drain = [&]() {
                __syncwarp();
                for (int base = 0; base < qcount; base += 32) {
                    const int e = base + lane;
                    bool pend = e < qcount;
                    const int r = pend ? (int)qr[e] : 32 + lane;  // idle lanes: distinct dummy rows
                    const uint64_t x = pend ? qk[e] : 0;
                    const unsigned grp = __match_any_sync(FULL, r);
                    unsigned todo = __ballot_sync(FULL, pend);
                    while (todo) {
                        const unsigned g = grp & todo;
                        if (pend && (g & (0u - g)) == (1u << lane)) {
                            heap_insert(heap + r * HS, m, x);
                            pend = false;
                        }
                        __syncwarp();
                        todo = __ballot_sync(FULL, pend);
                    }
                }
                qcount = 0;
                worst = fminf(__uint_as_float((uint32_t)(heap[lane * HS] >> 32)), seed_r);
                tq = fminf((worst - nq) + eps, tq_off);
            };

            // screened candidates waiting for their exact distance: ref position << 5 | row
            uint64_t *cq = cqbase + warp * CQCAP;
            int ccount = 0;
            // rescore queued candidates, one per lane (batches of 32; all of them when `all`, else
            // the whole batches, the rest moving to the front): the ref's exact coordinates and point
            // index from its tile record in global memory, the row's query coordinates, bound and
            // limit by shuffles from the lane that owns the row; survivors of the row's current bound
            // are queued as keys
            auto rescore = [&](bool all) {
                __syncwarp();
                const int n_do = all ? ccount : (ccount & ~31);
                for (int base = 0; base < n_do; base += 32) {
                    if (qcount > QCAP - 32) drain();
                    const int e = base + lane;
                    const bool has = e < n_do;
                    const uint64_t c = has ? cq[e] : 0;
                    const int r = (int)(c & 31u);
                    const int64_t jp = (int64_t)(c >> 5);  // the ref's position among the tiles
                    float qv[D];
#pragma unroll
                    for (int f = 0; f < D; ++f) qv[f] = __shfl_sync(FULL, qo[f], r);
                    const float worst_r = __shfl_sync(FULL, worst, r);
                    const long long limit_r = __shfl_sync(FULL, (long long)limit, r);
                    bool keep = false;
                    uint64_t key = 0;
                    if (has) {
                        const int col = (int)(jp & (RT - 1));
                        const unsigned char *rec = tiles_g + (jp / RT) * C::TILE_BYTES;
                        // the oracle's arithmetic: ((x0 - q0)^2 + (x1 - q1)^2) + ..., each step rounded
                        const float4 *rp4 = reinterpret_cast<const float4 *>(rec + C::OP_BYTES) + col * (C::DP / 4);
                        float rv[C::DP];
#pragma unroll
                        for (int f4 = 0; f4 < C::DP / 4; ++f4) {
                            const float4 t = __ldg(rp4 + f4);
                            rv[4 * f4] = t.x;
                            rv[4 * f4 + 1] = t.y;
                            rv[4 * f4 + 2] = t.z;
                            rv[4 * f4 + 3] = t.w;
                        }
                        int64_t jo = jp;  // index-order tiles: the position is the point index
                        if (pruned) {
                            if constexpr (C::IX_MODE == 1) jo = __float_as_int(rv[C::DP - 1]);
                            else if constexpr (C::IX_MODE == 2)
                                jo = __ldg(reinterpret_cast<const int32_t *>(rec + C::OP_BYTES + C::EX_BYTES) + col);
                            else jo = __ldg(ref_perm + jp);
                        }
                        const float t0 = sub_rn(rv[0], qv[0]);
                        float d2 = mul_rn(t0, t0);
#pragma unroll
                        for (int f = 1; f < D; ++f) {
                            const float tf = sub_rn(rv[f], qv[f]);
                            d2 = add_rn(d2, mul_rn(tf, tf));
                        }
                        keep = d2 <= worst_r && jo < (int64_t)limit_r;  // NaN never kept
                        key = (uint64_t)__float_as_uint(d2) << 32 | (uint32_t)jo;
                    }
                    const unsigned mk = __ballot_sync(FULL, keep);
                    if (keep) {
                        const int pos = qcount + __popc(mk & ((1u << lane) - 1u));
                        qk[pos] = key;
                        qr[pos] = (uint8_t)r;
                    }
                    qcount += __popc(mk);
                }
                const int rest = ccount - n_do;  // < 32
                __syncwarp();
                const uint64_t mv = lane < rest ? cq[n_do + lane] : 0;
                __syncwarp();
                if (lane < rest) cq[lane] = mv;
                __syncwarp();
                ccount = rest;
            };

            // the next stage's list entries are loaded one stage ahead (global loads that would
            // otherwise sit on the path from the accumulator to the screen)
            int64_t nx[C::TPS];
#pragma unroll
            for (int h = 0; h < C::TPS; ++h) nx[h] = (pruned && (uint32_t)h < ntiles) ? (int64_t)tl[h] : 0;
            for (uint32_t u = 0; u < nstg; ++u) {
                const uint32_t g = G + u;
                const uint32_t b = g % C::NBUF;
                const uint32_t t0 = u * C::TPS;                                  // the stage's first tile
                const int nh = (int)min((uint32_t)C::TPS, ntiles - t0);           // tiles in the stage
                int64_t j0[C::TPS];                                               // first ref position of each
#pragma unroll
                for (int h = 0; h < C::TPS; ++h) {
                    j0[h] = (pruned ? nx[h] : (int64_t)(tfirst + t0 + h)) * RT;
                    const uint32_t tn = t0 + C::TPS + h;
                    if (pruned && tn < ntiles) nx[h] = (int64_t)tl[tn];
                }
                const uint32_t tb = C::PAIR ? (uint32_t)qtw : b;  // this warp's accumulator barriers
                if (!mbar_wait_bounded(&t_full[tb], (g / C::NBUF) & 1, wait_ns)) aborted = true;
                if (__any_sync(FULL, aborted)) {
                    aborted = true;
                    break;
                }
                tc_fence_after();
                // 1) screen each tile of the stage: the minimum of each group of 8 columns (16 per row),
                //    the accumulator read in four 32-column chunks, each loading while the previous one
                //    is reduced; one vote per tile, since most tiles give no row of the warp a
                //    candidate.  A tile that does reads its passing chunks again (the accumulator is
                //    held until every tile of the stage is screened) for the candidate masks.
                uint32_t cmk[C::TPS][4];
                bool has_t[C::TPS];
#pragma unroll
                for (int h = 0; h < C::TPS; ++h) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) cmk[h][c] = 0u;
                    has_t[h] = false;
                    if (h >= nh) continue;  // warp-uniform
                    const uint32_t taddr =
                        tmem_base + ((uint32_t)(quad * 32) << 16) + b * C::BUF_COLS + qtw * C::RS + h * RT;
                    float gm[16];
                    auto group_mins = [&](const uint32_t (&v)[32], int c) {
#pragma unroll
                        for (int gi = 0; gi < 4; ++gi) {
#define NNGP_V(k) __uint_as_float(v[gi * 8 + (k)])
                            gm[c * 4 + gi] = fminf(min3f(NNGP_V(0), NNGP_V(1), NNGP_V(2)),
                                                   min3f(NNGP_V(3), NNGP_V(4), fminf(NNGP_V(5), fminf(NNGP_V(6), NNGP_V(7)))));
#undef NNGP_V
                        }
                    };
                    uint32_t va[32], vb[32];
                    tmem_ld32_nowait(taddr, va);
                    tmem_wait_ld(va);
                    tmem_ld32_nowait(taddr + 32, vb);
                    group_mins(va, 0);
                    tmem_wait_ld(vb);
                    tmem_ld32_nowait(taddr + 64, va);
                    group_mins(vb, 1);
                    tmem_wait_ld(va);
                    tmem_ld32_nowait(taddr + 96, vb);
                    group_mins(va, 2);
                    tmem_wait_ld(vb);
                    group_mins(vb, 3);
                    float cmin[4];  // minimum of each chunk
#pragma unroll
                    for (int c = 0; c < 4; ++c) cmin[c] = fminf(fminf(gm[4 * c], gm[4 * c + 1]), fminf(gm[4 * c + 2], gm[4 * c + 3]));
                    has_t[h] = __any_sync(FULL, fminf(fminf(cmin[0], cmin[1]), fminf(cmin[2], cmin[3])) < tq);
                    if (has_t[h]) {
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            if (__any_sync(FULL, cmin[c] < tq)) {  // warp-uniform: the load is collective
                                tmem_ld32_nowait(taddr + 32 * c, va);
                                tmem_wait_ld(va);
                                uint32_t cm = 0;
#pragma unroll
                                for (int gi = 0; gi < 4; ++gi) {
                                    if (gm[4 * c + gi] < tq) {  // only groups whose minimum passes
#pragma unroll
                                        for (int k = 0; k < 8; ++k)
                                            cm |= (__uint_as_float(va[gi * 8 + k]) < tq ? 1u : 0u) << (gi * 8 + k);
                                    }
                                }
                                cmk[h][c] = cm;
                            }
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&t_empty[tb]);
#pragma unroll
                for (int h = 0; h < C::TPS; ++h) {
                    if (!has_t[h]) continue;
                    {  // columns with j < limit only (pruned: positions < n_ref; the index test is per candidate)
                        const int64_t room = (pruned ? n_ref : limit) - j0[h];
                        if (room < RT) {
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                const int64_t r = room - c * 32;
                                if (r < 32) cmk[h][c] &= r <= 0 ? 0u : ((1u << (uint32_t)r) - 1u);
                            }
                        }
                    }
                    // 2) queue the tile's candidates (ref position, row): each lane walks its own
                    //    (column by column, chunks in order), one per warp iteration; whole batches of
                    //    32 are rescored as soon as they are queued
                    uint64_t lo = (uint64_t)cmk[h][0] | (uint64_t)cmk[h][1] << 32;
                    uint64_t hi = (uint64_t)cmk[h][2] | (uint64_t)cmk[h][3] << 32;
                    while (__any_sync(FULL, (lo | hi) != 0)) {
                        if (ccount > CQCAP - 32) rescore(false);
                        const bool has = (lo | hi) != 0;
                        int col = 0;
                        if (has) {
                            const bool use_lo = lo != 0;  // branch-free pick of the lowest remaining column
                            const uint64_t w = use_lo ? lo : hi;
                            col = __ffsll((long long)w) - 1 + (use_lo ? 0 : 64);
                            const uint64_t w2 = w & (w - 1);
                            lo = use_lo ? w2 : lo;
                            hi = use_lo ? hi : w2;
                        }
                        const unsigned mk = __ballot_sync(FULL, has);
                        if (has) cq[ccount + __popc(mk & ((1u << lane) - 1u))] = (uint64_t)(j0[h] + col) << 5 | (uint32_t)lane;
                        ccount += __popc(mk);
                    }
                }
                if (ccount >= 32) rescore(false);
                if (qcount >= DRAIN_AT) drain();
            }
            // write this warp's rows: each heap sorted ascending across the warp (bitonic, keys unique
            // except empty slots), index -1 for empty slots
            if (!aborted) {
                if (ccount > 0) rescore(true);
                if (qcount > 0) drain();
                __syncwarp();
                for (int rr = 0; rr < 32; ++rr) {
                    uint64_t x = lane < m ? heap[rr * HS + lane] : ~0ull;
#pragma unroll
                    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                        for (int jj = k >> 1; jj > 0; jj >>= 1) {
                            const uint64_t o = __shfl_xor_sync(FULL, x, jj);
                            const bool take_min = ((lane & jj) == 0) == ((lane & k) == 0);
                            x = take_min ? (o < x ? o : x) : (o > x ? o : x);
                        }
                    }
                    const int64_t rq = C::PAIR ? rr * EPI_WARPS + warp : warp * 32 + rr;  // item row of row rr
                    if (out_slot >= 0) {
                        items.partial[((int64_t)out_slot * C::ROWS + rq) * 32 + lane] = x;
                    } else if (rq < n_item_rows && lane < m) {
                        out[(point_of(q0 + rq) - out_base) * m + lane] = (int32_t)(uint32_t)x;  // out_base: shard's first row
                    }
                }
            }
        }
        g_tile += nstg;
        ++it;
        if (aborted) *s_abort = 1;
        __syncthreads();
    }

    // teardown: report a timeout, let copies and MMAs this CTA issued finish (bounded by the
    // full kWaitLimitNs whatever wait_ns is), free TMEM
    if ((aborted || *s_abort) && threadIdx.x == 0) flag_or(flags, NNGP_FLAG_TIMEOUT);
    if ((C::TMA_WARP ? copy_warp : producer_warp) && lane == 0 && (aborted || *s_abort)) {
        // copies issued but never waited for: let them land before the CTA's shared memory goes.
        // With TMA_WARP the copying thread does not know which ones the MMA thread waited for; the
        // last S it issued are the latest uses of their stages (earlier ones were waited for before
        // their stage was refilled), and a wait on a phase that has completed returns at once.
        const uint32_t g_from = C::TMA_WARP ? (tma_issued > (uint32_t)S ? tma_issued - S : 0u) : tma_landed;
        for (uint32_t g = g_from; g < tma_issued; ++g) mbar_wait_bounded(&b_full[g % S], (g / S) & 1);
    }
    if (producer_warp && lane == 0 && (aborted || *s_abort)) {
        // MMAs in flight: a commit tracks every earlier tcgen05 operation of this thread, so the
        // phase of the last committed tile covers them all (a tile whose MMAs were never issued
        // has no phase to wait for: g_tile counts an aborted item's stages in full)
        if (last_tf >= 0) mbar_wait_bounded(&t_full[last_tf], last_tf_par);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (producer_warp) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(C::TMEM_COLS));
    }
}

// Self-test of the UMMA operand layout: D = A B^T for A, B given row-major (128 x KP), through
// the same shared-memory layout, descriptors, tcgen05.mma and tcgen05.ld path as the search
// (TF32 operands, or BF16 operands converted from A and B when BF16).
template <int KP, bool BF16 = false>
__global__ void __launch_bounds__(THREADS) tc_layout_selftest_kernel(const float *__restrict__ a,
                                                                    const float *__restrict__ b,
                                                                    float *__restrict__ d,
                                                                    int32_t *__restrict__ flags) {
    constexpr int ESZ = BF16 ? 2 : 4;
    constexpr int KMMA = BF16 ? 16 : 8;
    constexpr bool SW = KP * ESZ == 128;  // the search's choice for the same shape
    __shared__ __align__(1024) unsigned char sA[QT * KP * ESZ];
    __shared__ __align__(1024) unsigned char sB[RT * KP * ESZ];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int e = threadIdx.x; e < QT * KP; e += blockDim.x) {
        if constexpr (BF16) *reinterpret_cast<uint16_t *>(sA + op_offset<2, SW>(e / KP, e % KP, QT)) = bf16_bits(a[e]);
        else *reinterpret_cast<float *>(sA + op_offset<4, SW>(e / KP, e % KP, QT)) = a[e];
    }
    for (int e = threadIdx.x; e < RT * KP; e += blockDim.x) {
        if constexpr (BF16) *reinterpret_cast<uint16_t *>(sB + op_offset<2, SW>(e / KP, e % KP, RT)) = bf16_bits(b[e]);
        else *reinterpret_cast<float *>(sB + op_offset<4, SW>(e / KP, e % KP, RT)) = b[e];
    }
    fence_proxy_async_smem();
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(kSelftestCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_slot;
    if (warp == 4 && lane == 0) {
#pragma unroll
        for (int i = 0; i < KP / KMMA; ++i)
            mma_op<BF16>(tmem_base, op_desc<SW, ESZ, KMMA>(smem_addr(sA), QT, i),
                         op_desc<SW, ESZ, KMMA>(smem_addr(sB), RT, i), i > 0 ? 1u : 0u);
        mma_commit(&bar);
    }
    const bool ok = mbar_wait_bounded(&bar, 0);
    if (!ok && threadIdx.x == 0) flag_or(flags, NNGP_FLAG_TIMEOUT);
    tc_fence_after();
    if (warp < 4 && ok) {
        uint32_t v[32];
        for (int c = 0; c < RT / 32; ++c) {
            tmem_ld32_nowait(tmem_base + ((uint32_t)(warp * 32) << 16) + c * 32, v);
            tmem_wait_ld(v);
            for (int k = 0; k < 32; ++k) d[(warp * 32 + lane) * RT + c * 32 + k] = __uint_as_float(v[k]);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 4) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kSelftestCols));
    }
}

// d 12 and 16 fill an SM with one CTA: two query tiles per work item give it 8 epilogue warps
// and halve the ref-tile stream per query
template <int D, int QTILES = (D == 12 || D == 16) ? 2 : 1> TcVariant tc_make() {
    using C = Cfg<D, QTILES>;
    TcVariant v;
    v.fn = knn_tc_kernel<D, QTILES>;
    v.build = build_tc_tiles_kernel<D>;
    v.smem = C::SMEM;
    v.stage_bytes = C::TILE_BYTES;  // bytes of a tile record in global memory
    v.dp = C::DP;
    v.ctas_per_sm = C::CTAS_PER_SM;
    v.threads = C::THREADS;
    v.rows_per_item = C::ROWS;
    return v;
}

}  // namespace tc

tc::TcVariant tc_variant(int D, int M) {
    if (M > tc::LIST) return tc::TcVariant{};
    switch (D) {
        case 1: return tc::tc_make<1>();
        case 2: return tc::tc_make<2>();
        case 3: return tc::tc_make<3>();
        case 4: return tc::tc_make<4>();
        case 5: return tc::tc_make<5>();
        case 6: return tc::tc_make<6>();
        case 7: return tc::tc_make<7>();
        case 8: return tc::tc_make<8>();
        case 12: return tc::tc_make<12>();
        case 16: return tc::tc_make<16>();
        case 20: return tc::tc_make<20>();
        case 24: return tc::tc_make<24>();
    }
    return tc::TcVariant{};
}

}  // namespace nngp

extern "C" nngp_status nngp_tc_layout_selftest(const float *a, const float *b, int32_t kp, float *d, int32_t *flags,
                                               void *stream) {
    using namespace nngp;
    set_error("");
    if (!a || !b || !d) return fail(NNGP_ERR_INVALID_ARGUMENT, "tc_layout_selftest: null pointer");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (kp) {
        case 8: tc::tc_layout_selftest_kernel<8><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        case 16: tc::tc_layout_selftest_kernel<16><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        case 32: tc::tc_layout_selftest_kernel<32><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        default: return fail(NNGP_ERR_UNSUPPORTED, "tc_layout_selftest: kp must be 8, 16 or 32");
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

extern "C" nngp_status nngp_tc_layout_selftest_bf16(const float *a, const float *b, int32_t kp, float *d,
                                                    int32_t *flags, void *stream) {
    using namespace nngp;
    set_error("");
    if (!a || !b || !d) return fail(NNGP_ERR_INVALID_ARGUMENT, "tc_layout_selftest_bf16: null pointer");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (kp) {
        case 16: tc::tc_layout_selftest_kernel<16, true><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        case 32: tc::tc_layout_selftest_kernel<32, true><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        case 64: tc::tc_layout_selftest_kernel<64, true><<<1, tc::THREADS, 0, st>>>(a, b, d, flags); break;
        default: return fail(NNGP_ERR_UNSUPPORTED, "tc_layout_selftest_bf16: kp must be 16, 32 or 64");
    }
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}
