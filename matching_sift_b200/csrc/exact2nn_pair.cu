// Exact 2-NN search kernel on CTA pairs (tcgen05 cta_group::2).
//
// Same arithmetic, pruning and outputs as exact2nn_u8_kernel (exact2nn.cu);
// this kernel only changes how the tensor cores are fed. A cluster of two
// CTAs on the two SMs of a TPC issues M = 256 MMAs: each CTA keeps its own
// 128 query rows of a 256-row "pair tile" in shared memory and loads half
// (64 rows) of every 128-row base tile; the leader CTA issues one
// 256 x 128 x 32 MMA per K step and the accumulator rows land in the TMEM of
// the CTA that owns them. Compared with single-CTA 128 x 128 MMAs this halves
// the base bytes every SM streams per MMA, and it leaves room in TMEM for two
// accumulator buffers per query tile, so the MMA of the next base tile runs
// while the epilogue is still scanning the previous one.
//
// Per CTA: QPT query tiles x 128 rows (a work group of the pair = 2 * QPT
// * 128 queries; QPT = 2 gives the single-CTA kernel's groups of 512), TMEM
// 2 * QPT slots x 128 columns = (query tile, buffer); unit n uses buffer n % 2.
// QB query buffers: with 2 the next group's queries load while the current
// group's MMAs run (batches of small problems change groups often).
//
// Work: a list of problems (WorkItem: query rows, base rows, unit range); a
// single search is a list of one. Units (problem, query group, base tile) are
// numbered problem by problem and every CTA pair owns a contiguous range; all
// roles walk the same range with a Cursor.
//
// Warp roles (96 + 32 * 8 * QPT threads per CTA):
//   warp 0       TMA producer (both CTAs): its own query rows, its half of
//                each base tile (completion counted on the leader's barrier)
//                and the full norms record of the tile (local barrier)
//   warp 1       TMEM allocator (both CTAs); MMA issuer of the even units
//                (leader CTA only)
//   warps 2..    epilogue (both CTAs): warp w owns query tile (w - 2) / 8,
//                buffer ((w - 2) / 4) % 2 (so it scans every other unit, all
//                128 columns) and TMEM lane quarter w % 4
//   last warp    MMA issuer of the odd units (leader CTA only)
//
// MMA issue: on sm_100a every mbarrier test and every tcgen05.commit costs
// the issuing thread on the order of a hundred cycles, against 64 cycles per
// 256 x 128 x 32 MMA, and one thread issuing every unit (8 MMAs, two barrier
// tests, a commit) left the tensor pipe idle half of the time. Two issuer
// threads, each owning one accumulator buffer (unit parity), share the work;
// each tests its next unit's barriers behind its queued MMAs and commits once
// per unit.
//
// Barriers and who signals them (L = only the leader's copy is used):
//   full[s]    (L) both CTAs' base halves of stage s landed        TMA tx
//   rfull[s]   norms record of stage s landed (per CTA)            TMA tx
//   sfree[s]   the 8 epilogue warps that scanned stage s's unit are
//              done: its MMAs completed (they waited on tfull) and its
//              record is no longer read (per CTA)                  arrive
//   qfull[b]   (L) query tiles of both CTAs landed in buffer b      TMA tx
//   qempty[b]  MMAs of the group in query buffer b done (both CTAs) commit x 2 (one per issuer), multicast
//   tfull[sl]  accumulators of TMEM slot sl = (query tile t, buffer b) done
//              (one commit per tile, so a tile's epilogue starts
//              before the next tile's MMAs finish)                commit, multicast
//   tempty[sl] (L) the 4 warps of slot sl in each CTA read it: the
//              issuer's next MMAs into that tile start without
//              waiting for the other tile's epilogue              remote arrive
// Every wait is bounded (2 s); an expired wait raises the CTA's abort flag
// and records an error code, and every role still reaches the teardown.
//
// Instantiations of one body:
//   exact2nn_u8_pair_kernel   u8 rows (128 B), kind::i8, s32 accumulators,
//                             4 MMAs of K = 32 per 128 x 128 tile product
//   exact2nn_f16_pair_kernel  FP16 rows (256 B = two 128-byte K blocks, each
//                             loaded by its own TMA box of 64 halves), kind::f16
//                             with f32 accumulators, 8 MMAs of K = 16. This is
//                             the counterpart of the reference's half GEMM
//                             (cublasHgemm, src/knn_brute.cu:262-266). Values
//                             are integers times 2^-s (|integer| <= 255), so
//                             every product and partial sum is an integer
//                             multiple of 2^-2s below 2^24 * 2^-2s and the f32
//                             accumulators are exact. The epilogue prunes on
//                             the raw f32 bits (non-negative values order like
//                             int32) and converts to the u8 kernel's integer
//                             dot products (times dscale = 2^2s, rounded) only
//                             the subgroup maxima and the values of passing
//                             subgroups; the rest is shared.
//   exact2nn_u8_pair_batch_kernel<QPT, QB>  u8 batches with the shapes the
//                             batch autotuner chooses from.
#include <climits>
#include "exact2nn.cuh"
#include "ptx.cuh"
#include "epilogue.cuh"

namespace sift {

namespace {

constexpr int kPHalf = kBN / 2;                  // base rows loaded per CTA per unit
constexpr int kPRecBytes = kRecInts * 4;         // 640 B
constexpr uint16_t kPairMask = 0x3;
constexpr size_t kPSmemBudget = 225 * 1024;

// Element formats of the instantiations.
enum PairMode : int {
    kModeU8 = 0,     // u8 rows, kind::i8, integer keys
    kModeF16Int = 1, // FP16 rows holding integers x 2^-s, kind::f16, integer keys
    kModeFloat = 2,  // split FP16 rows [hi | lo] (or plain FP16 rows), kind::f16, float keys
    kModeU8Fold = 3, // u8 rows plus a fifth MMA that folds the norms in (fold_records_kernel)
};

// Shapes of one instantiation. A row of 128 elements is kKBlocks blocks of
// 128 bytes (split rows: 2 hi blocks then 2 lo blocks); each block of a tile
// is stored as its own SW128 K-major tile (rows x 128 B), and every MMA
// consumes 32 bytes of K.
template <int MODE, int QPT, int QB>
struct PairCfg {
    static constexpr bool F16 = MODE == kModeF16Int || MODE == kModeFloat;
    static constexpr bool kFold = MODE == kModeU8Fold;
    static constexpr int kFoldStage = kFold ? kFoldHalfBytes : 0;  // digits of the base half, per stage
    static constexpr int kAConst = kFold ? kBM * 32 : 0;           // the constant fold row, 128 rows
    static constexpr int kElemBytes = F16 ? 2 : 1;
    static constexpr int kKBlocks = !F16 ? 1 : (MODE == kModeFloat ? 4 : 2);
    static constexpr int kBoxElems = 128 / kElemBytes;       // TMA box width of one K block
    static constexpr int kQKBlock = kBM * 128;               // bytes of one K block of a query tile
    static constexpr int kBKBlock = kPHalf * 128;            // bytes of one K block of a base half
    static constexpr int kQTileBytes = kKBlocks * kQKBlock;  // 16 / 32 KB
    static constexpr int kQBufBytes = QPT * kQTileBytes;
    static constexpr int kBHalfBytes = kKBlocks * kBKBlock;  // 8 / 16 KB
    static constexpr int kSlots = 2 * QPT;                   // (query tile, buffer)
    static constexpr int kEpiWarps = 4 * kSlots;             // one per (slot, lane quarter)
    static constexpr int kMma2Warp = 2 + kEpiWarps;          // second MMA issuer (odd units)
    static constexpr int kThreads = 64 + 32 * kEpiWarps + 32;
    static constexpr int kTmemCols = kSlots * kBN;
    static constexpr int kStagesFit =
        static_cast<int>((kPSmemBudget - 1024 - 512 - QB * kQBufBytes - kAConst) /
                         (kBHalfBytes + kFoldStage + kPRecBytes));
    // 16 stages when they fit (a power of two keeps the ring index cheap in
    // the issue loop), else as many as fit.
    static constexpr int kStages = kStagesFit >= 16 ? 16 : kStagesFit;
    struct __align__(8) Ctl {
        uint64_t full[kStages];
        uint64_t rfull[kStages];
        uint64_t sfree[kStages];
        uint64_t qfull[QB], qempty[QB];
        uint64_t tfull[2 * QPT], tempty[2 * QPT];  // per TMEM slot (tile t, buffer b) = 2 t + b
        uint64_t drain;
        uint32_t tmem_base;
        int abort_flag;
        int no_abort;
    };
    static constexpr size_t kSmemBytes =
        1024 + QB * kQBufBytes + kStages * (kBHalfBytes + kFoldStage) + kAConst + kStages * kPRecBytes +
        sizeof(Ctl);
    // M = 256 (the pair), N = kBN; s32 accumulators for u8 x u8, f32 for f16 x f16.
    static constexpr uint32_t kIdesc =
        F16 ? ptx::idesc_make(1 /*F32*/, 0 /*F16*/, 0 /*F16*/, 2 * kBM, kBN)
            : ptx::idesc_make(2 /*S32*/, 0 /*u8*/, 0 /*u8*/, 2 * kBM, kBN);
    static_assert(kStages >= 4, "base ring too shallow");
    static_assert(kSmemBytes <= 227 * 1024, "shared memory");
    static_assert(kSmemBytes <= kPSmemBudget + 1024, "shared memory budget");
};

// Walks a CTA pair's contiguous unit range over the work items.
struct Cursor {
    const WorkItem* items;  // device list, or null for the single item `it`
    int n_items;
    WorkItem it;            // current problem
    int p, g, j;            // problem, query group, base tile

    __device__ __forceinline__ void init(const WorkItem* list, int n, const WorkItem& single, long long w) {
        items = list;
        n_items = n;
        p = 0;
        if (list) {
            int lo = 0, hi = n - 1;  // largest p with u_begin <= w (empty items share the next one's u_begin)
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (list[mid].u_begin <= w) lo = mid; else hi = mid - 1;
            }
            p = lo;
            it = list[p];
        } else {
            it = single;
        }
        const long long r = w - it.u_begin;
        g = it.tiles > 0 ? static_cast<int>(r / it.tiles) : 0;
        j = static_cast<int>(r - static_cast<long long>(g) * it.tiles);
    }
    __device__ __forceinline__ bool last_of_group() const { return j + 1 == it.tiles; }
    // One unit forward; true when the next unit opens a query group.
    __device__ __forceinline__ bool next() {
        if (++j < it.tiles) return false;
        j = 0;
        if (++g < it.groups) return true;
        g = 0;
        if (items) {
            while (++p < n_items) {
                it = items[p];
                if (it.groups > 0 && it.tiles > 0) break;
            }
        }
        return true;
    }
    __device__ __forceinline__ long long group_first_unit() const {
        return it.u_begin + static_cast<long long>(g) * it.tiles;
    }
};

// has_lo (kModeFloat only): the rows carry lo blocks (split float rows); when
// false they are plain FP16 rows and only the hi.hi products are formed.
// TWO_PASS: the two-pass epilogue (single searches) or the one-pass scan
// (batches of small problems).
template <int MODE, int QPT, int QB, bool TWO_PASS>
__device__ __forceinline__ void pair_body(const CUtensorMap& qmap, const CUtensorMap& bmap, const CUtensorMap& fmap,
                                          const int32_t* __restrict__ brec, const ExactPlan& plan,
                                          const WorkItem* __restrict__ items, int n_items, const WorkItem& single,
                                          int4* __restrict__ partial, int32_t* __restrict__ thresh,
                                          int* __restrict__ err, float dscale, bool has_lo = false) {
    using Cfg = PairCfg<MODE, QPT, QB>;
    constexpr bool F16 = Cfg::F16;
    // K blocks actually loaded per row (split rows without lo parts: the hi blocks only).
    const int kb_load = (MODE == kModeFloat && !has_lo) ? 2 : Cfg::kKBlocks;
    constexpr int kPStages = Cfg::kStages;
    constexpr int kPQTileBytes = Cfg::kQTileBytes;
    constexpr int kPBHalfBytes = Cfg::kBHalfBytes;
    constexpr int kPEpiWarps = Cfg::kEpiWarps;
    using PairCtl = typename Cfg::Ctl;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_u32 & 1023u)) & 1023u);
    uint8_t* q_smem = smem;
    uint8_t* b_smem = smem + QB * Cfg::kQBufBytes;
    uint8_t* f_smem = b_smem + kPStages * kPBHalfBytes;        // fold digits per stage (fold only)
    uint8_t* a_smem = f_smem + kPStages * Cfg::kFoldStage;     // the constant fold row tile (fold only)
    int32_t* r_smem = reinterpret_cast<int32_t*>(a_smem + Cfg::kAConst);
    PairCtl* ctl = reinterpret_cast<PairCtl*>(r_smem + kPStages * kRecInts);
    const uint32_t q_s = ptx::smem_u32(q_smem);
    const uint32_t b_s = ptx::smem_u32(b_smem);
    const uint32_t r_s = ptx::smem_u32(r_smem);
    const uint32_t f_s = ptx::smem_u32(f_smem);
    const uint32_t a_s = ptx::smem_u32(a_smem);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = ptx::cluster_ctarank();
    const bool leader = rank == 0;
    const int pair = static_cast<int>(blockIdx.x >> 1);
    const long long W = plan.units;
    const long long G = plan.grid;  // pairs
    const long long w_begin = plan_w0(pair, W, G);
    const int n_units = static_cast<int>(plan_w0(pair + 1, W, G) - w_begin);

    const uint32_t bar_full = ptx::smem_u32(&ctl->full[0]);
    const uint32_t bar_rfull = ptx::smem_u32(&ctl->rfull[0]);
    const uint32_t bar_sfree = ptx::smem_u32(&ctl->sfree[0]);
    const uint32_t bar_qfull = ptx::smem_u32(&ctl->qfull[0]);
    const uint32_t bar_qempty = ptx::smem_u32(&ctl->qempty[0]);
    const uint32_t bar_tfull = ptx::smem_u32(&ctl->tfull[0]);
    const uint32_t bar_tempty = ptx::smem_u32(&ctl->tempty[0]);
    const uint32_t bar_drain = ptx::smem_u32(&ctl->drain);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPStages; ++s) {
            ptx::mbar_init(bar_full + 8 * s, 1);
            ptx::mbar_init(bar_rfull + 8 * s, 1);
            ptx::mbar_init(bar_sfree + 8 * s, kPEpiWarps / 2);
        }
        for (int b = 0; b < QB; ++b) {
            ptx::mbar_init(bar_qfull + 8 * b, 1);
            ptx::mbar_init(bar_qempty + 8 * b, 2);  // one commit per MMA issuer
        }
        for (int sl = 0; sl < 2 * QPT; ++sl) {
            ptx::mbar_init(bar_tfull + 8 * sl, 1);
            ptx::mbar_init(bar_tempty + 8 * sl, 2 * 4);  // the 4 warps of the slot in each CTA
        }
        ptx::mbar_init(bar_drain, 2);
        ctl->abort_flag = 0;
        ctl->no_abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) {
        ptx::tmem_alloc_pair(ptx::smem_u32(&ctl->tmem_base), Cfg::kTmemCols);
        ptx::tmem_relinquish_pair();
    }
    if constexpr (Cfg::kFold) {
        // The constant fold row a = {1, 16, 255 x 30} for all 128 query rows,
        // in the no-swizzle K-major layout of fold_records_kernel's digits
        // (8-row groups of 256 B, two 16-byte K chunks 128 B apart).
        for (int i = threadIdx.x; i < Cfg::kAConst / 4; i += blockDim.x) {
            const int kc = (i >> 5) & 1, b0 = (i & 3) * 4;  // 4 bytes: K = 16 kc + b0 .. + 3
            uint32_t word = 0;
            #pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int k = 16 * kc + b0 + b;
                word |= static_cast<uint32_t>(k == 0 ? 1 : (k == 1 ? 16 : 255)) << (8 * b);
            }
            reinterpret_cast<uint32_t*>(a_smem)[i] = word;
        }
        ptx::fence_proxy_async();
    }
    ptx::tc_fence_before();
    __syncthreads();
    // Both CTAs' barriers are initialised before any cross-CTA signal.
    ptx::cluster_sync();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    volatile int* abort_flag = &ctl->abort_flag;
    volatile int* never = &ctl->no_abort;

    Cursor cur;
    if (n_units > 0) cur.init(items, n_items, single, w_begin);

    if (warp == 0) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer
            ptx::tma_prefetch_desc(&qmap);
            ptx::tma_prefetch_desc(&bmap);
            const uint32_t lead_qfull = ptx::mapa(bar_qfull, 0);
            const uint32_t lead_full = ptx::mapa(bar_full, 0);
            int ngroups = 0;
            bool new_group = true;
            int n = 0;
            for (; n < n_units; ++n) {
                if (new_group) {
                    const int qb = ngroups % QB;
                    if (ngroups >= QB && !ptx::mbar_wait_cluster(bar_qempty + 8 * qb, ((ngroups / QB) - 1) & 1,
                                                                 abort_flag, err, kErrWaitQuery))
                        break;
                    if (leader) ptx::mbar_arrive_expect_tx(bar_qfull + 8 * qb, 2 * QPT * kb_load * Cfg::kQKBlock);
                    for (int t = 0; t < QPT; ++t) {
                        const int row = cur.it.a_off + ((cur.g * QPT + t) * 2 + static_cast<int>(rank)) * kBM;
                        #pragma unroll
                        for (int kb = 0; kb < Cfg::kKBlocks; ++kb)
                            if (kb < kb_load)
                                ptx::tma_load_2d_pair(
                                    q_s + qb * Cfg::kQBufBytes + t * kPQTileBytes + kb * Cfg::kQKBlock, &qmap,
                                    kb * Cfg::kBoxElems, row, lead_qfull + 8 * qb);
                    }
                    ++ngroups;
                }
                const int s = n % kPStages;
                if (!ptx::mbar_wait(bar_sfree + 8 * s, ((n / kPStages) & 1) ^ 1, abort_flag, err, kErrWaitProducer))
                    break;
                if (leader) ptx::mbar_arrive_expect_tx(bar_full + 8 * s, 2 * (kb_load * Cfg::kBKBlock + Cfg::kFoldStage));
                const int brow = cur.it.b_off + cur.j * kBN + static_cast<int>(rank) * kPHalf;
                #pragma unroll
                for (int kb = 0; kb < Cfg::kKBlocks; ++kb)
                    if (kb < kb_load)
                        ptx::tma_load_2d_pair(b_s + s * kPBHalfBytes + kb * Cfg::kBKBlock, &bmap, kb * Cfg::kBoxElems,
                                              brow, lead_full + 8 * s);
                if constexpr (Cfg::kFold)
                    ptx::tma_load_2d_pair(f_s + s * Cfg::kFoldStage, &fmap, 0,
                                          ((cur.it.rec_off + cur.j) * 2 + static_cast<int>(rank)) * 8, lead_full + 8 * s);
                ptx::mbar_arrive_expect_tx(bar_rfull + 8 * s, kPRecBytes);
                ptx::bulk_load(r_s + s * kPRecBytes, brec + static_cast<size_t>(cur.it.rec_off + cur.j) * kRecInts,
                               kPRecBytes, bar_rfull + 8 * s);
                new_group = cur.next();
            }
            // Drain: this CTA's copies land before it may exit. Records are
            // counted locally; base halves are consumed once the epilogue
            // has released the stage; query buffers once their MMAs are done.
            for (int k = (n > kPStages ? n - kPStages : 0); k < n; ++k) {
                ptx::mbar_wait(bar_rfull + 8 * (k % kPStages), (k / kPStages) & 1, never, err, kErrWaitDrain);
                ptx::mbar_wait(bar_sfree + 8 * (k % kPStages), (k / kPStages) & 1, never, err, kErrWaitDrain);
            }
            for (int k = (ngroups > QB ? ngroups - QB : 0); k < ngroups; ++k)
                ptx::mbar_wait_cluster(bar_qempty + 8 * (k % QB), (k / QB) & 1, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else if (warp == 1 || warp == Cfg::kMma2Warp) {
        if (lane == 0 && leader) {
            // ------------------------------------------------- MMA issuers
            // Thread mt issues the units n with n % 2 == mt (accumulator
            // buffer mt); both walk every unit to follow the query groups.
            const int mt = warp == 1 ? 0 : 1;
            constexpr uint32_t idesc = Cfg::kIdesc;
            constexpr int kMaxProd = MODE == kModeFloat ? 6 : Cfg::kKBlocks;
            const int n_prod = MODE == kModeFloat ? (has_lo ? 6 : 2) : Cfg::kKBlocks;
            const uint64_t b_desc0 = ptx::sdesc_sw128(b_s);
            int ngroups = 0;
            bool new_group = true;
            uint64_t a_desc0 = ptx::sdesc_sw128(q_s);
            int qb = 0;
            bool pre_full = ptx::mbar_test_wait(bar_full + 8 * (mt % kPStages), 0);
            bool pre_tempty = ptx::mbar_test_wait(bar_tempty + 8 * mt, 1);
            for (int n = 0; n < n_units; ++n) {
                if (new_group) {
                    qb = ngroups % QB;
                    if (!ptx::mbar_wait_cluster(bar_qfull + 8 * qb, (ngroups / QB) & 1, abort_flag, err, kErrWaitQuery))
                        break;
                    a_desc0 = ptx::sdesc_sw128(q_s + qb * Cfg::kQBufBytes);
                    ++ngroups;
                }
                if ((n & 1) == mt) {
                    const int s = n % kPStages;
                    if (!pre_full &&
                        !ptx::mbar_wait_cluster(bar_full + 8 * s, (n / kPStages) & 1, abort_flag, err, kErrWaitMmaFull))
                        break;
                    const uint32_t tpar_free = ((n >> 1) & 1) ^ 1;
                    const uint64_t b_desc = b_desc0 + static_cast<uint64_t>((s * kPBHalfBytes) >> 4);
                    bool ok = true;
                    #pragma unroll
                    for (int t = 0; t < QPT; ++t) {
                        // Each tile's slot is handed back on its own: the tile's MMAs
                        // start as soon as its epilogue warps release it.
                        if (!(t == 0 && pre_tempty) &&
                            !ptx::mbar_wait_cluster(bar_tempty + 8 * (t * 2 + mt), tpar_free, abort_flag, err,
                                                    kErrWaitMmaTmem)) {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t d = tmem + (t * 2 + mt) * kBN;
                        // K-block products: (kb, kb) for every block of the row;
                        // split float rows: hi.hi for both K halves, then (with lo
                        // parts) hi.lo' and lo.hi'.
                        #pragma unroll
                        for (int p = 0; p < kMaxProd; ++p) {
                            if (p >= n_prod) break;
                            const int ab = MODE == kModeFloat ? (p < 4 ? (p & 1) : 2 + (p & 1)) : p;
                            const int bb = MODE == kModeFloat ? (p < 2 ? p : (p < 4 ? 2 + (p & 1) : (p & 1))) : p;
                            const uint64_t a_desc =
                                a_desc0 + static_cast<uint64_t>((t * kPQTileBytes + ab * Cfg::kQKBlock) >> 4);
                            const uint64_t b_kb = b_desc + static_cast<uint64_t>((bb * Cfg::kBKBlock) >> 4);
                            #pragma unroll
                            for (int kk = 0; kk < 4; ++kk) {
                                const uint32_t acc = (p > 0 || kk > 0) ? 1u : 0u;
                                if constexpr (F16)
                                    ptx::mma_f16_pair(d, a_desc + 2 * kk, b_kb + 2 * kk, idesc, acc);
                                else
                                    ptx::mma_i8_pair(d, a_desc + 2 * kk, b_kb + 2 * kk, idesc, acc);
                            }
                        }
                        if constexpr (Cfg::kFold)
                            ptx::mma_i8_pair(d, ptx::sdesc_kmajor_noswz(a_s, 128, 256),
                                             ptx::sdesc_kmajor_noswz(f_s + s * Cfg::kFoldStage, 128, 256),
                                             ptx::idesc_make(2 /*S32*/, 0 /*u8*/, 1 /*s8*/, 2 * kBM, kBN), 1u);
                        ptx::tc_commit_pair_mc(bar_tfull + 8 * (t * 2 + mt), kPairMask);
                    }
                    if (!ok) break;
                    // Test the barriers of this issuer's next unit (n + 2) behind its queued MMAs.
                    if (n + 2 < n_units) {
                        pre_full = ptx::mbar_test_wait(bar_full + 8 * ((n + 2) % kPStages), ((n + 2) / kPStages) & 1);
                        pre_tempty = ptx::mbar_test_wait(bar_tempty + 8 * mt, (((n + 2) >> 1) & 1) ^ 1);  // tile 0
                    }
                }
                // Both issuers release the query buffer at the end of a group
                // (each commit covers that issuer's own MMAs).
                if (n + 1 == n_units || cur.last_of_group()) ptx::tc_commit_pair_mc(bar_qempty + 8 * qb, kPairMask);
                new_group = cur.next();
            }
            // Drain: all issued MMAs complete before TMEM is released.
            ptx::tc_commit_pair(bar_drain);
            ptx::mbar_wait(bar_drain, 0, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ epilogue
        const int e = warp - 2;
        const int t = e >> 3;             // query tile of this warp
        const int buf = (e >> 2) & 1;     // accumulator buffer = parity of the units this warp scans
        const int quarter = warp & 3;     // TMEM lane quarter this warp may access
        const uint32_t taddr = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + (t * 2 + buf) * kBN;
        const int slot = t * 2 + buf;     // TMEM slot and its barriers
        const uint32_t lead_tempty = ptx::mapa(bar_tempty + 8 * slot, 0);
        Top2 st{INT_MAX, -1, INT_MAX, -1, INT_MAX};
        int published = INT_MAX;
        int split = 0, q = 0;
        bool active = false, valid = false, open = false;
        bool new_group = true;
        // The query's shared bound is read one unit of this warp ahead: the
        // value used for unit n was loaded while unit n - 2 was scanned, so
        // the L2 round trip never waits in front of the first chunk. An older
        // value is still a valid bound (bounds only decrease).
        int next_thr = INT_MAX;

        for (int n = 0; n < n_units; ++n) {
            if (new_group) {
                if (open && valid)
                    partial[(static_cast<size_t>(split) * 2 + buf) * plan.q_pad + q] =
                        make_int4(st.k1, st.i1, st.k2, st.i2);
                st = Top2{INT_MAX, -1, INT_MAX, -1, INT_MAX};
                published = INT_MAX;
                open = true;
                const int q_local = ((cur.g * QPT + t) * 2 + static_cast<int>(rank)) * kBM + quarter * 32 + lane;
                valid = q_local < cur.it.n_a;
                active = __any_sync(0xffffffffu, valid);
                split = pair - plan_cta_of(cur.group_first_unit(), W, G);
                q = cur.it.a_off + q_local;
                next_thr = valid ? __ldcg(thresh + q) : INT_MAX;
            }
            const int j = cur.j;
            if ((n & 1) == buf) {
                const int shared_thr = next_thr;
                next_thr = valid ? __ldcg(thresh + q) : INT_MAX;
                const int s = n % kPStages;
                const uint32_t rpar = (n / kPStages) & 1, tpar = (static_cast<uint32_t>(n) >> 1) & 1;
                // Both tests are issued back to back so their latencies overlap.
                const bool r_ok = ptx::mbar_try_wait(bar_rfull + 8 * s, rpar);
                const bool t_ok = ptx::mbar_try_wait_cluster(bar_tfull + 8 * slot, tpar, 0u);
                bool waited = true;
                if (!r_ok) waited = ptx::mbar_wait(bar_rfull + 8 * s, rpar, abort_flag, err, kErrWaitEpilogue);
                if (waited && !t_ok)
                    waited = ptx::mbar_wait_cluster(bar_tfull + 8 * slot, tpar, abort_flag, err, kErrWaitEpilogue);
                if (!__all_sync(0xffffffffu, waited)) break;
                ptx::tc_fence_after();
                if (active) {
                    st.thr = min(st.thr, shared_thr);
                    const int32_t* rec = r_smem + s * kRecInts;
                    constexpr int kKind = MODE == kModeFloat ? kAccFloat : (F16 ? kAccF32Int : kAccS32);
                    const int row0 = cur.it.idx_base + j * kBN;
                    if constexpr (TWO_PASS) {
                        // Two passes over the slot's 128 columns (8 chunks of 16).
                        // The first bounds every 8-row subgroup against the
                        // threshold held at its start, with no vote and no branch,
                        // while chunk c + 1 loads; the second forms exact keys
                        // only in chunks where some lane's bound passed, reading
                        // them from the slot again (still held). Then the slot is
                        // handed back.
                        uint32_t va[16], vb[16];
                        const int thr0 = st.thr;
                        const int vt = -((thr0 >> 1) + (thr0 & 1));  // fold variant: -floor((thr0 + 1) / 2)
                        auto bits = [&](const uint32_t (&v)[16], int c) -> uint32_t {
                            if constexpr (Cfg::kFold)
                                return fold_bits16(v, vt);
                            else
                                return bound16<kKind>(v, rec + kBN + 2 * c, thr0, dscale);
                        };
                        uint32_t pass = 0;  // bit 2 c + k: subgroup k of chunk c may hold a candidate
                        ptx::tmem_ld16(taddr, va);
                        ptx::tmem_ld_wait(va);
                        #pragma unroll
                        for (int c = 1; c < 8; c += 2) {
                            ptx::tmem_ld16(taddr + 16 * c, vb);
                            pass |= bits(va, c - 1) << (2 * (c - 1));
                            ptx::tmem_ld_wait(vb);
                            if (c + 1 < 8) {
                                ptx::tmem_ld16(taddr + 16 * (c + 1), va);
                                pass |= bits(vb, c) << (2 * c);
                                ptx::tmem_ld_wait(va);
                            }
                        }
                        pass |= bits(vb, 7) << 14;
                        // Subgroups in increasing order, so the top-2 still sees
                        // the rows in index order (ties keep the lower index).
                        uint32_t todo = __reduce_or_sync(0xffffffffu, pass);
                        while (todo) {
                            const int g = __ffs(todo) - 1;
                            todo &= todo - 1;
                            uint32_t v8[8];
                            ptx::tmem_ld8(taddr + 8 * g, v8);
                            ptx::tmem_ld_wait(v8);
                            if ((pass >> g) & 1u) exact8<kKind>(v8, row0 + 8 * g, rec + 8 * g, st, dscale);
                        }
                        ptx::tc_fence_before();
                        __syncwarp();
                        if (lane == 0) ptx::mbar_arrive_cluster_relaxed(lead_tempty);
                    } else {
                        // One pass (batches: their bounds pass often, so exact
                        // keys are formed at once from the registers): chunk c + 1
                        // loads while chunk c is scanned, and the slot is handed
                        // back as soon as the last chunk is in registers.
                        uint32_t va[16], vb[16];
                        auto scan = [&](const uint32_t (&v)[16], int c) {
                            scan16<kKind>(v, row0 + 16 * c, rec + 16 * c, rec + kBN + 2 * c, st, dscale);
                        };
                        ptx::tmem_ld16(taddr, va);
                        ptx::tmem_ld_wait(va);
                        #pragma unroll
                        for (int c = 1; c < 8; c += 2) {
                            ptx::tmem_ld16(taddr + 16 * c, vb);
                            scan(va, c - 1);
                            ptx::tmem_ld_wait(vb);
                            if (c + 1 < 8) {
                                ptx::tmem_ld16(taddr + 16 * (c + 1), va);
                                scan(vb, c);
                                ptx::tmem_ld_wait(va);
                            }
                        }
                        ptx::tc_fence_before();
                        __syncwarp();
                        if (lane == 0) ptx::mbar_arrive_cluster_relaxed(lead_tempty);
                        scan(vb, 7);
                    }
                    if (valid && st.k2 < published) {
                        atomicMin(thresh + q, st.k2);
                        published = st.k2;
                    }
                } else {
                    ptx::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) ptx::mbar_arrive_cluster_relaxed(lead_tempty);
                }
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(bar_sfree + 8 * s);
            }
            new_group = cur.next();
        }
        if (open && valid)
            partial[(static_cast<size_t>(split) * 2 + buf) * plan.q_pad + q] = make_int4(st.k1, st.i1, st.k2, st.i2);
    }

    ptx::tc_fence_before();
    __syncthreads();
    // The leader's MMAs into this CTA's TMEM are drained and no CTA of the
    // pair signals the other after this point.
    ptx::cluster_sync();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc_pair(tmem, Cfg::kTmemCols);
    }
}

using CfgU8 = PairCfg<kModeU8, 2, 1>;
using CfgF16 = PairCfg<kModeF16Int, 2, 1>;
using CfgFold = PairCfg<kModeU8Fold, 2, 1>;
// Split float rows are 512 bytes: one query tile per CTA (groups of 256
// queries) leaves room for 4 base stages.
using CfgFloat = PairCfg<kModeFloat, 1, 1>;

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CfgU8::kThreads, 1)
    exact2nn_u8_pair_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                            const int32_t* __restrict__ brec, const ExactPlan plan, const WorkItem single,
                            int4* __restrict__ partial, int32_t* __restrict__ thresh, int* __restrict__ err) {
    pair_body<kModeU8, 2, 1, true>(qmap, bmap, qmap, brec, plan, nullptr, 1, single, partial, thresh, err, 1.0f);
}

// fmap: the folding digits (fold_records_kernel), a 2-D u8 tensor of
// 256-byte rows, 8 rows per half tile.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CfgFold::kThreads, 1)
    exact2nn_u8fold_pair_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                                const __grid_constant__ CUtensorMap fmap, const int32_t* __restrict__ brec,
                                const ExactPlan plan, const WorkItem single, int4* __restrict__ partial,
                                int32_t* __restrict__ thresh, int* __restrict__ err) {
    pair_body<kModeU8Fold, 2, 1, true>(qmap, bmap, fmap, brec, plan, nullptr, 1, single, partial, thresh, err, 1.0f);
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CfgF16::kThreads, 1)
    exact2nn_f16_pair_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                             const int32_t* __restrict__ brec, const ExactPlan plan, const WorkItem single,
                             int4* __restrict__ partial, int32_t* __restrict__ thresh, int* __restrict__ err,
                             float dscale) {
    pair_body<kModeF16Int, 2, 1, true>(qmap, bmap, qmap, brec, plan, nullptr, 1, single, partial, thresh, err,
                                       dscale);
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CfgFloat::kThreads, 1)
    exact2nn_float_pair_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                               const int32_t* __restrict__ brec, const ExactPlan plan, const WorkItem single,
                               int4* __restrict__ partial, int32_t* __restrict__ thresh, int* __restrict__ err,
                               int has_lo) {
    pair_body<kModeFloat, 1, 1, true>(qmap, bmap, qmap, brec, plan, nullptr, 1, single, partial, thresh, err, 1.0f,
                                      has_lo != 0);
}

template <int QPT, int QB>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PairCfg<kModeU8, QPT, QB>::kThreads, 1)
    exact2nn_u8_pair_batch_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                                  const int32_t* __restrict__ brec, const ExactPlan plan,
                                  const WorkItem* __restrict__ items, int n_items, int4* __restrict__ partial,
                                  int32_t* __restrict__ thresh, int* __restrict__ err) {
    pair_body<kModeU8, QPT, QB, false>(qmap, bmap, qmap, brec, plan, items, n_items, WorkItem{}, partial, thresh, err,
                                       1.0f);
}

template <typename K>
cudaError_t set_smem_once(K kernel, size_t bytes, bool (&done)[64]) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !done[dev]) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) done[dev] = true;
    }
    return cudaSuccess;
}

WorkItem single_item(const ExactPlan& plan) {
    WorkItem w{};
    w.a_off = 0;
    w.n_a = plan.q_n;
    w.b_off = 0;
    w.n_b = plan.r_n;
    w.u_begin = 0;
    w.groups = plan.q_groups;
    w.tiles = plan.base_tiles;
    w.rec_off = 0;
    return w;
}

template <int QPT, int QB>
cudaError_t launch_batch_variant(const CUtensorMap& qmap, const CUtensorMap& bmap, const int32_t* brec,
                                 const BatchPlan& bp, int4* partial, int32_t* thresh, int* err, cudaStream_t stream) {
    using Cfg = PairCfg<kModeU8, QPT, QB>;
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_u8_pair_batch_kernel<QPT, QB>, Cfg::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (bp.plan.grid <= 0) return cudaSuccess;
    exact2nn_u8_pair_batch_kernel<QPT, QB><<<2 * bp.plan.grid, Cfg::kThreads, Cfg::kSmemBytes, stream>>>(
        qmap, bmap, brec, bp.plan, bp.items, bp.n_items, partial, thresh, err);
    return cudaGetLastError();
}

}  // namespace

size_t exact2nn_pair_smem_bytes() { return CfgU8::kSmemBytes; }

cudaError_t launch_exact2nn_u8_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                    const ExactPlan& plan, int4* partial, int32_t* thresh, int* err,
                                    cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_u8_pair_kernel, CfgU8::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_u8_pair_kernel<<<2 * plan.grid, CfgU8::kThreads, CfgU8::kSmemBytes, stream>>>(
        qmap, bmap_half, brec, plan, single_item(plan), partial, thresh, err);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_u8fold_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half,
                                        const CUtensorMap& fmap, const int32_t* brec, const ExactPlan& plan,
                                        int4* partial, int32_t* thresh, int* err, cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_u8fold_pair_kernel, CfgFold::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_u8fold_pair_kernel<<<2 * plan.grid, CfgFold::kThreads, CfgFold::kSmemBytes, stream>>>(
        qmap, bmap_half, fmap, brec, plan, single_item(plan), partial, thresh, err);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_u8fold_pair_item(const CUtensorMap& qmap, const CUtensorMap& bmap_half,
                                             const CUtensorMap& fmap, const int32_t* brec, const ExactPlan& plan,
                                             const WorkItem& item, int4* partial, int32_t* thresh, int* err,
                                             cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_u8fold_pair_kernel, CfgFold::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_u8fold_pair_kernel<<<2 * plan.grid, CfgFold::kThreads, CfgFold::kSmemBytes, stream>>>(
        qmap, bmap_half, fmap, brec, plan, item, partial, thresh, err);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_u8_pair_item(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                         const ExactPlan& plan, const WorkItem& item, int4* partial, int32_t* thresh,
                                         int* err, cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_u8_pair_kernel, CfgU8::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_u8_pair_kernel<<<2 * plan.grid, CfgU8::kThreads, CfgU8::kSmemBytes, stream>>>(
        qmap, bmap_half, brec, plan, item, partial, thresh, err);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_f16_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                     const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, float dscale,
                                     cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_f16_pair_kernel, CfgF16::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_f16_pair_kernel<<<2 * plan.grid, CfgF16::kThreads, CfgF16::kSmemBytes, stream>>>(
        qmap, bmap_half, brec, plan, single_item(plan), partial, thresh, err, dscale);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_float_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                       const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, bool has_lo,
                                       cudaStream_t stream) {
    static bool attr_set[64] = {};
    cudaError_t e = set_smem_once(exact2nn_float_pair_kernel, CfgFloat::kSmemBytes, attr_set);
    if (e != cudaSuccess) return e;
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_float_pair_kernel<<<2 * plan.grid, CfgFloat::kThreads, CfgFloat::kSmemBytes, stream>>>(
        qmap, bmap_half, brec, plan, single_item(plan), partial, thresh, err, has_lo ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_u8_pair_batch(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                          const BatchPlan& bp, int4* partial, int32_t* thresh, int* err, int qpt,
                                          int qbuf, cudaStream_t stream) {
    if (qpt == 2 && qbuf == 1) return launch_batch_variant<2, 1>(qmap, bmap_half, brec, bp, partial, thresh, err, stream);
    if (qpt == 2 && qbuf == 2) return launch_batch_variant<2, 2>(qmap, bmap_half, brec, bp, partial, thresh, err, stream);
    if (qpt == 1 && qbuf == 2) return launch_batch_variant<1, 2>(qmap, bmap_half, brec, bp, partial, thresh, err, stream);
    return cudaErrorInvalidValue;
}

}  // namespace sift
