// Host-side declarations of the kernel launchers (plain pointers and sizes).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "comb_windows.h"

namespace vkzg {

struct Fr;
struct Fp;
struct G1A;
struct G1J;

constexpr int kBlobElems = 4096;
constexpr int kExtElems = 8192;
constexpr int kCells = 128;        // cells per blob = proofs per blob = circulant size
constexpr int kCellElems = 64;     // field elements per cell = terms per phase-A output
constexpr int kDigits = 32;        // signed 8-bit windows per scalar
constexpr int kLadderDigits = 16;  // doubled ladder rows; phase B reads slots d >= 16 as phi images
constexpr int kBuckets = 128;      // |digit| in 1..128
constexpr int kHalf = 64;
constexpr size_t kBlobBytes = 131072;
constexpr size_t kProofBytes = 48;
constexpr size_t kCellBytes = 2048;
constexpr size_t kPositionPoints = (size_t)kCells * kCellElems * kDigits; // 262144

// Phase B's convolution parts.  The 128-point cyclic convolution of a blob's
// u[j] with the fixed taps is split by `levels` radix-2 folds (points
// v[j] +- v[j + m], taps (t[e] +- t[e + m]) / 2): one cyclic part of
// 128 >> levels points at slots [0, 128 >> levels) and, for each level l, a
// negacyclic part of 128 >> l points at slots [128 >> l, 128 >> (l - 1)).
// Plans 0-2 use one level (the two halves); plans 3-4 kPartLevels.
constexpr int kFBMaxParts = 4;
constexpr int kPartLevels = 3;
struct PartLayout {
    int n;                          // levels + 1
    uint32_t size[kFBMaxParts];     // outputs = points = taps of the part
    uint32_t off[kFBMaxParts];      // first slot; its tap items start at item 32 * off
    uint32_t nega[kFBMaxParts];     // 1: negacyclic
};
inline PartLayout part_layout(int levels) {
    PartLayout L{};
    L.n = levels + 1;
    L.size[0] = (uint32_t)kCells >> levels;
    L.off[0] = 0;
    L.nega[0] = 0;
    for (int q = 1; q <= levels; q++) {
        const int l = levels + 1 - q;
        L.size[q] = (uint32_t)kCells >> l;
        L.off[q] = (uint32_t)kCells >> l;
        L.nega[q] = 1;
    }
    return L;
}

// Pair sums shared by the buckets of a part (plans 3-4): when the same pair of
// tap items -- rows a and b of the ladder, taps e and e + delta, relative sign
// s -- falls into two or more buckets of a part, the part's outputs share
//   M[x] = L_a[x] + s L~_b[x - delta],   x < n,
// (L~ the ladder row extended cyclically or negacyclically like the part), and
// each such pair becomes one tap item (e, digit slot 32 + t, sign of the first):
// M~ obeys the same extension rule, so it is read like a ladder row.
constexpr int kMaxPartTypes = 256 - kDigits; // digit slots 32..255
struct DerivType {
    uint8_t part, row_a, row_b, neg; // neg: s = -1
    uint32_t delta;                  // 0 <= delta < n
    uint32_t base;                   // first point of M in a blob's derived array
};

// Round structure of plan 3's phase B (see build_flatb_plan): per round r and
// part q, each bucket's list length, element offsets, pair offsets and odd
// buckets, identical for every output of a part.
constexpr int kFBMaxRounds = 12;
struct FlatBPlan {
    int rounds;
    PartLayout parts;
    uint32_t stride[kFBMaxRounds + 1];                    // elements per output in round r's buffer
    uint32_t pairs[kFBMaxRounds][kFBMaxParts];            // pairs per output
    uint32_t n_odd[kFBMaxRounds][kFBMaxParts];
    uint32_t cnt[kFBMaxRounds + 1][kFBMaxParts][kBuckets];
    uint32_t base[kFBMaxRounds + 1][kFBMaxParts][kBuckets + 1];
    uint32_t pscan[kFBMaxRounds][kFBMaxParts][kBuckets + 1];
    uint8_t odd[kFBMaxRounds][kFBMaxParts][kBuckets];
    uint32_t n_empty[kFBMaxParts];              // buckets no tap digit reaches, per part
    uint8_t empty[kFBMaxParts][kBuckets];
};
bool build_flatb_plan(const PartLayout &parts, const uint32_t offsets[][kBuckets + 1], FlatBPlan &plan);

// Setup-derived device tables (immutable once built).
struct DeviceTables {
    G1A *pos = nullptr;             // [128 j][64 i][32 d] affine, 2^(8d) X[j][i]
    Fr *roots_fwd = nullptr;        // w_8192^i
    Fr *roots_inv = nullptr;        // w_8192^-i
    uint32_t *tap_items[2] = {nullptr, nullptr};  // e | d<<8 | neg<<16, grouped by bucket
    uint32_t *tap_offsets[2] = {nullptr, nullptr}; // [129]
    uint32_t *tap_perm[2] = {nullptr, nullptr};    // [128] buckets by descending load
    Fr *shift_fwd = nullptr;        // 7^k / 8192                (recovery)
    Fr *shift_inv = nullptr;        // 7^-k / 8192 / R           (recovery; output lands canonical)
    Fr *inv_blob_r2 = nullptr;      // [1] (1/4096) in Montgomery form
    uint32_t *part_items = nullptr;   // plans 3-4: tap items of the kPartLevels parts, part q from 32 * off[q]
    uint32_t *part_offsets = nullptr; // [kFBMaxParts][129]
    DerivType *deriv = nullptr;       // plans 3-4: the shared pair sums
    uint16_t *deriv_of = nullptr;     // [deriv_points] type of each derived point
    uint32_t deriv_points = 0;        // derived points per blob
    int deriv_types = 0;
    uint32_t deriv_base[kFBMaxParts] = {}; // first derived point of part q (type t: + t n_q)
    FlatBPlan *fb_plan = nullptr;   // plan 3's phase-B rounds
    int fb_rounds = 0;              // 0: plan 3 uses the per-warp phase B
    uint32_t fb_stride[2] = {0, 0}; // elements per output after rounds 1 and 2
};

// Per-batch working set for proofs, capacity `cap` blobs.
struct ProofWork {
    uint8_t *blobs = nullptr;   // [cap][131072]
    Fr *coeffs = nullptr;       // [cap][4096] Montgomery
    Fr *scalars = nullptr;      // [cap][128 j][64 i] canonical
    G1J *buckets = nullptr;     // [cap][128][128]
    G1J *points = nullptr;      // [cap][128] reduce outputs
    G1J *ladder = nullptr;      // [cap][128][16] 2^(8d) v[j] of the folded parts
    G1A *ladder_aff = nullptr;  // [cap][128][32]: d < 16 the ladder, d >= 16 its phi images
    G1A *deriv_buf = nullptr;   // plans 3-4: [cap][deriv_points] shared pair sums
    uint8_t *proofs = nullptr;  // [cap][128][48]
    uint32_t *err = nullptr;    // [cap]
    // batch-affine accumulation (plans 1, 2)
    G1A *bucket_aff = nullptr;  // [cap][128][128] affine bucket sums
    G1A *ba_scratch = nullptr;  // [ba_blocks][kBAScratchPoints]
    int ba_blocks = 0;          // persistent grid size of the batch-affine kernels
    uint32_t *task_ctr = nullptr; // [2] next task of phase A / phase B (zeroed before phase A)
    const G1A *comb = nullptr;    // plan 3: digit table [128 j][64 i][entries of D windows], shared by provers
    int comb_windows = 0;         // its windows per scalar (CombWindows)
    // plan 3's grid-wide tree rounds (flat_sizes gives the sizes)
    int16_t *flat_dig = nullptr;  // [cap * 128][64 D] digits
    G1A *flat_buf[2] = {nullptr, nullptr};
    uint32_t *flat_pre = nullptr;
    Fp *flat_others = nullptr, *flat_tot = nullptr, *flat_totinv = nullptr;
    size_t flat_slots = 0;
    int flat_blocks = 0;
    G1A *flatb_buf[2] = {nullptr, nullptr}; // phase B's round buffers
    int plan = 1;               // 0 serial Jacobian; 1 batch-affine + binary-split reduction; 2 batch-affine + serial reduction
    G1A *red_scratch = nullptr; // [cap * 128][247] batch-affine reduction slots
    // plans 3-4: the grid-wide rounds of each phase as one cooperative launch
    // (grid barriers between passes) when true, else three launches per round
    bool coop = false;
    uint32_t *sync = nullptr;   // [4] grid-barrier words of the cooperative launches
};
// Batch-affine kernels: VKZG_BA_THREADS threads per block, one warp sums the
// buckets of kWarpOutputs MSM outputs at a time.  Per-warp scratch: round-1 and
// round-2 outputs (at most 1088 and 608 points per output of 2048 points in 128
// buckets), prefix products (32 pairs x 12 words per lane per output = 512
// points), and phase A's sorted bucket items (2048 x 2 bytes per output, 43
// points).
#ifndef VKZG_BA_THREADS
#define VKZG_BA_THREADS 256
#endif
#ifndef VKZG_WARP_OUTPUTS
#define VKZG_WARP_OUTPUTS 4
#endif
constexpr int kWarpOutputs = VKZG_WARP_OUTPUTS;
constexpr int kBAWarpScratchPoints = kWarpOutputs * (1088 + 608 + 512 + 43);
constexpr int kBAScratchPoints = (VKZG_BA_THREADS / 32) * kBAWarpScratchPoints; // per block

struct RecoverWork {
    uint8_t *cells = nullptr;     // [cap][8192*32]
    uint8_t *present = nullptr;   // [cap][128]
    uint8_t *out = nullptr;       // [cap][8192*32]
    uint32_t *err = nullptr;      // [cap] more than 64 cells missing
};

// Proof pipeline over `n` blobs already resident in w.blobs.
cudaError_t launch_proofs(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s);
// Recovery pipeline over `n` blobs already resident in w.cells / w.present.
cudaError_t launch_recover(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s);
// Table generation from 4096 compressed monomial points already on the device.
// Writes t.pos; needs `scratch` of at least setup_scratch_bytes().
size_t setup_scratch_bytes();
size_t comb_build_scratch_bytes(int windows);
constexpr int kCombMinWindows = 18, kCombMaxWindows = 32;
// Bytes per digit-table entry: an affine point (96 bytes), or with
// VKZG_COMB_ENTRY_BYTES=128 a point padded to one 128-byte line, so that a
// random gather touches one line instead of straddling two half of the time.
// Measured at 256 blobs, 13-bit window: phase A 12.79 ms padded against 12.82
// unpadded (the first round's gathers are prefetched one pair ahead and hidden
// behind the products), for a third more table memory: unpadded by default.
#ifndef VKZG_COMB_ENTRY_BYTES
#define VKZG_COMB_ENTRY_BYTES 96
#endif
constexpr size_t kCombEntryBytes = VKZG_COMB_ENTRY_BYTES;
static_assert(kCombEntryBytes == 96 || kCombEntryBytes == 128, "an entry is a point, or a point padded to a line");
struct FlatSizes {
    int blocks = 0;
    size_t lanes = 0, dig = 0, buf0 = 0, buf1 = 0, slots = 0, pre_words = 0;
};
FlatSizes flat_sizes(int cap, int windows);
int launch_tree_sums(const G1A *lists, int n_lists, uint32_t m, G1A *buf0, G1A *buf1, uint32_t *pre, Fp *others,
                     Fp *tot, Fp *totinv, size_t slots, int blocks, G1A *sums, cudaStream_t s);
cudaError_t launch_comb_table(const DeviceTables &t, G1A *comb, void *scratch, int windows, cudaStream_t s);
cudaError_t launch_setup_tables(const uint8_t *d_g1_monomial, G1A *pos, const Fr *roots_fwd, void *scratch,
                                uint32_t *d_err, cudaStream_t s);
cudaError_t configure_kernels();
}
struct vkzg_prover;
namespace vkzg {
void adopt_tuning(vkzg_prover *dst, const vkzg_prover *src);
// the cooperative forms of plans 3-4 fit blocks_per_sm blocks per SM
bool coop_supported(int blocks_per_sm);
// no cooperative launches for this prover (a serving lane: several lanes'
// pipelines run at once, and each cooperative launch wants the whole GPU)
void disable_coop(vkzg_prover *p);
// frees the buffers none of a fully tuned prover's plans uses (before any capture)
void trim_working_set(vkzg_prover *p);
// digit-table byte budget of a prover (before its first tuning)
void set_comb_budget(vkzg_prover *p, uint64_t bytes);
void precapture_graphs(vkzg_prover *p, uint32_t max_n);

// process-wide count of kernels launched by the launchers above
void count_launches(int k);
uint64_t launches_total();

} // namespace vkzg
