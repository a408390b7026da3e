// C ABI of include/vkzg.h and include/vkzg_b200.h over the CUDA kernels.
//
// Reference counterpart: src/vkzg.cpp (Vulkan instance, pipelines, buffers and
// the per-call command buffer).  Here a prover owns one CUDA stream, the setup
// tables resident in device memory, and a working set sized for
// max_batch_size blobs; each API call copies a chunk in, launches the stage
// kernels on the stream, and copies the chunk out.  Calls on one prover are
// serialised by a mutex (src/vkzg.cpp:1188,1206).
#include "../../include/vkzg.h"
#include "../../include/vkzg_b200.h"
#include "device_util.cuh"
#include "glv.h"
#include "kernels.h"

#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <map>
#include <thread>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

using namespace vkzg;

namespace vkzg {
cudaError_t configure_proof_kernels();
cudaError_t configure_recover_kernels();
cudaError_t configure_cells_kernels();
int batch_affine_blocks_per_sm();
size_t reduce_scratch_points(int cap_blobs);
cudaError_t launch_proofs_timed(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s,
                                cudaEvent_t *ev, bool skip_front = false);
cudaError_t launch_proofs_front(const DeviceTables &t, const ProofWork &w, int off, int cnt, cudaStream_t s);
cudaError_t launch_recover_timed(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s,
                                 cudaEvent_t *ev);

static std::atomic<uint64_t> g_launches{0};
static thread_local uint64_t t_launches = 0; // this thread's share (graph captures count their launches by it)
void count_launches(int k) {
    g_launches.fetch_add((uint64_t)(int64_t)k, std::memory_order_relaxed);
    t_launches += (uint64_t)(int64_t)k;
}
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
} // namespace vkzg

static constexpr int kProofStages = 10;
static constexpr int kRecoverStages = 1;
static const char *kProofStageNames[kProofStages] = {"blob_to_coeffs", "circulant", "phase_a",  "reduce_a",
                                                     "fold",           "ladder",    "normalize", "phase_b",
                                                     "reduce_b",       "finish"};
static const char *kRecoverStageNames[kRecoverStages] = {"recover"};

// Plan 3's digit table (proof_kernels.cu, k_phase_a_comb): tens of GB, built
// on first use and shared by every prover of the process on the same device
// with the same setup tables; freed with the last of them.
struct CombTable {
    int device = 0;
    int windows = 0; // per scalar (CombWindows)
    G1A *d = nullptr;
    size_t bytes = 0;
    double build_ms = 0.0;
    ~CombTable() {
        if (!d) return;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        cudaFree(d);
        cudaSetDevice(cur);
    }
};

struct vkzg_prover {
    int device = 0;
    std::string name;
    uint32_t sm_count = 0;
    std::string tables_source;
    cudaStream_t stream = nullptr;
    std::mutex mutex;
    DeviceTables t;
    std::vector<std::pair<void *, size_t>> allocs;
    uint32_t cap = 0;
    ProofWork pw;
    RecoverWork rw;
    uint32_t *h_err = nullptr; // pinned, cap words
    bool timing = false;
    cudaEvent_t ev[kProofStages + 1] = {};
    cudaEvent_t ev_rec[kRecoverStages + 1] = {};
    cudaEvent_t ev_in = nullptr, ev_out = nullptr; // stream handshakes of the device-pointer API
    // stage times: filled after a blocking call, or lazily (pending_kind) after
    // a device-pointer call once the caller has synchronised
    mutable double last_proof_ms[kProofStages] = {};
    mutable double last_recover_ms[kRecoverStages] = {};
    mutable bool pending_proof = false, pending_recover = false;
    // autotuner: plan per power-of-two chunk size (see choose_plan)
    int plan_forced = -1;
    std::map<uint32_t, int> plan_of;
    std::map<uint32_t, std::array<double, 5>> plan_ms;
    std::string tables_id;            // identity of the setup tables, for sharing the digit table
    std::shared_ptr<CombTable> comb;  // plan 3's digit table, once built
    bool comb_failed = false, flat_failed = false;
    // device memory: everything this prover allocated (tables_bytes of it the
    // setup tables); the shared digit table is counted apart, in comb->bytes
    uint64_t dev_bytes = 0, tables_bytes = 0;
    // digit table: byte budget ($VKZG_COMB_BUDGET_GB, default 20 GiB; a serving
    // loop passes its own), the window count the tuner chose (0 = not yet), and
    // the count the phase-A round buffers are sized for (they serve any smaller)
    uint64_t comb_budget = 20ull << 30;
    bool coop_off = false; // see vkzg::disable_coop
    bool trimmed = false;  // see vkzg::trim_working_set: only the tuned plans' buffers are left
    uint32_t plan0_cap = 0; // blobs the Jacobian bucket array holds once trimmed
    int comb_windows_chosen = 0, comb_buf_windows = 0;
    struct WindowTrial {
        int windows;
        uint64_t bytes;
        double build_ms, ms;
    };
    std::map<uint32_t, std::vector<WindowTrial>> window_trials; // per tuned size class
    // CUDA graphs of the proof pipeline per (chunk size, plan), see run_proofs
    struct GraphRec {
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
    };
    std::map<uint64_t, GraphRec> graphs;
    bool use_graphs = true;
    // side streams for host-buffer chunks, so that copies in, kernels and copies
    // out overlap: a recovery or cells chunk of kPartsFrom blobs or more runs as
    // parts of at least kRecPartBlobs blobs (32 parts at 256 blobs: 116 k blobs/s
    // of recovery through the C ABI; 8-blob parts beat 16- and 32-blob parts by
    // 4-6 %; splitting from 16 blobs rather than 64 took recovery of 32 blobs from
    // 0.62 to 0.52 ms and cells of 48 blobs from 0.60 to 0.52 ms), each copying in,
    // computing and copying out on side stream (part mod kSides); a proof chunk
    // uploads in kUploadPieces pieces (2 beat 4, 8 and 16: each piece adds a
    // launch of the per-blob front that fills only part of the GPU)
    static constexpr int kSides = 16;
    static constexpr uint32_t kRecPartBlobs = 8, kRecMaxParts = 32, kPartsFrom = 16;
    static constexpr int kUploadPieces = 2;
    cudaStream_t side[kSides] = {};
    cudaEvent_t side_ev[kSides + 1] = {};
    cudaEvent_t part_ev[kRecMaxParts] = {}; // a part's copy out done (pageable recovery)
    std::string tune_cache;
    cudaEvent_t ev_tune[2] = {nullptr, nullptr};
    // Pinned staging for callers' pageable host buffers (allocated on the first
    // call that passes one, cap x 256 KB each way).  A pageable buffer is copied
    // by host threads into (or out of) it part by part, so that those copies,
    // the DMA on the side streams and the kernels of other parts overlap; the
    // driver's own staging of pageable copies runs one copy at a time
    // (measured: 13 k recovery blobs/s at 256 blobs from pageable buffers).
    uint8_t *stage_in = nullptr, *stage_out = nullptr;
    size_t stage_bytes = 0;

    ~vkzg_prover() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto &x : side)
            if (x) cudaStreamSynchronize(x);
        if (stage_in) cudaFreeHost(stage_in);
        if (stage_out) cudaFreeHost(stage_out);
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.exec);
        for (auto &x : side)
            if (x) cudaStreamDestroy(x);
        for (auto &e : side_ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : part_ev)
            if (e) cudaEventDestroy(e);
        for (auto &a : allocs) cudaFree(a.first);
        if (h_err) cudaFreeHost(h_err);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : ev_rec)
            if (e) cudaEventDestroy(e);
        if (ev_in) cudaEventDestroy(ev_in);
        for (auto &e : ev_tune)
            if (e) cudaEventDestroy(e);
        if (ev_out) cudaEventDestroy(ev_out);
        if (stream) cudaStreamDestroy(stream);
    }
    template <typename T>
    bool alloc(T *&ptr, size_t count) {
        void *p = nullptr;
        if (cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) return false;
        allocs.push_back({p, count * sizeof(T) + 16});
        dev_bytes += count * sizeof(T) + 16;
        ptr = reinterpret_cast<T *>(p);
        return true;
    }
    // frees one allocation made by alloc (the stream must be idle)
    template <typename T>
    void release(T *&ptr) {
        for (auto it = allocs.begin(); it != allocs.end(); ++it)
            if (it->first == (void *)ptr) {
                cudaFree(it->first);
                dev_bytes -= it->second;
                allocs.erase(it);
                break;
            }
        ptr = nullptr;
    }
};

// ------------------------------------------------------------------ utils

const char *vkzg_error_string(vkzg_result r) {
    switch (r) {
    case VKZG_OK: return "ok";
    case VKZG_ERR_BADARGS: return "invalid argument";
    case VKZG_ERR_MALLOC: return "allocation failed";
    case VKZG_ERR_IO: return "i/o error";
    case VKZG_ERR_SETUP: return "malformed trusted setup";
    case VKZG_ERR_GPU: return "gpu error";
    case VKZG_ERR_INVALID_BLOB: return "blob contains a non-canonical field element";
    }
    if (r == VKZG_B200_PENDING) return "request still in flight (wait timed out)";
    return "unknown error";
}

void vkzg_options_default(vkzg_options *opts) {
    if (opts) opts->max_batch_size = 0;
}

const char *vkzg_prover_device_name(const vkzg_prover *p) { return p ? p->name.c_str() : ""; }
uint32_t vkzg_prover_gpu_core_count(const vkzg_prover *p) { return p ? p->sm_count : 0; }
const char *vkzg_b200_prover_tables_source(const vkzg_prover *p) { return p ? p->tables_source.c_str() : ""; }

// --------------------------------------------------------- host-side tables
namespace {

std::string library_dir() {
    Dl_info info;
    if (dladdr((void *)&vkzg_prover_new, &info) && info.dli_fname) {
        std::string s(info.dli_fname);
        const size_t k = s.rfind('/');
        if (k != std::string::npos) return s.substr(0, k);
    }
    return ".";
}

// w_8192 = 7^((r-1)/8192) and its powers (the reference's roots tables,
// src/precomputed_tables.cpp:43-44)
void host_roots(std::vector<Fr> &fwd, std::vector<Fr> &inv) {
    // (r-1)/8192
    const uint32_t e[8] = {0xfff80000u, 0xdff7ffffu, 0x2017fff2u, 0xc02a9dedu,
                           0xc0404d0eu, 0xea4199ceu, 0x3a994cebu, 0x00039f6du};
    const Fr w = fr_pow_words(fr_from_u32(7), e, 8);
    const Fr wi = fr_inv(w);
    fwd.resize(kExtElems);
    inv.resize(kExtElems);
    fwd[0] = inv[0] = fr_one();
    for (int i = 1; i < kExtElems; i++) {
        fwd[i] = fr_mul(fwd[i - 1], w);
        inv[i] = fr_mul(inv[i - 1], wi);
    }
}

// c[e] = (1/128) sum_{t<64} w_128^(e t), e < 128: the taps of the 128-point
// cyclic convolution phase B computes (src/precomputed_tables.cpp:45-49).
static void host_taps128(const std::vector<Fr> &fwd, Fr c[kCells]) {
    const Fr inv128 = fr_inv(fr_from_u32(128));
    for (int e = 0; e < kCells; e++) {
        Fr acc = fr_zero();
        for (int t = 0; t < kHalf; t++) acc = fr_add(acc, fwd[((e * t) % kCells) * (kExtElems / kCells)]);
        c[e] = fr_mul(acc, inv128);
    }
}

// Signed base-256 digits of one tap (Montgomery form).  With split_phi the tap
// is k1 + k2 z^2 (glv.h): slots 0..15 hold k1's digits (applied to 2^(8d) L),
// slots 16..31 the digits of -k2 (applied to 2^(8d) phi(L)); without it, the
// reference's 32 digits of the full tap.  False if a split does not fit its
// 16 digits (it always does).
static bool tap_digits(const Fr &tap, bool split_phi, int dig[kDigits]) {
    const Fr can = fr_to_canonical(tap);
    if (split_phi) {
        const GlvSplit sp = glv_split(can.v);
        return glv_digits(sp.mag[0], sp.neg[0], dig) && glv_digits(sp.mag[1], sp.neg[1], dig + kGlvDigits);
    }
    int carry = 0;
    for (int d = 0; d < kDigits; d++) {
        int v = (int)((can.v[d >> 2] >> ((d & 3) * 8)) & 0xffu) + carry;
        carry = 0;
        if (v > kBuckets) {
            v -= 2 * kBuckets;
            carry = 1;
        }
        dig[d] = v;
    }
    return true;
}

// Items e | d << 8 | neg << 16 of n_taps taps grouped by bucket |digit| - 1,
// bucket offsets, and the buckets by descending load (the reference's
// kernel_items / offsets / perm layout).
static void group_items(const int (*dig)[kDigits], int n_taps, uint32_t *items, uint32_t offsets[kBuckets + 1],
                        uint32_t perm[kBuckets]) {
    uint32_t count[kBuckets] = {0};
    for (int e = 0; e < n_taps; e++)
        for (int d = 0; d < kDigits; d++)
            if (dig[e][d]) count[abs(dig[e][d]) - 1]++;
    uint32_t acc = 0;
    for (int k = 0; k < kBuckets; k++) {
        offsets[k] = acc;
        acc += count[k];
    }
    offsets[kBuckets] = acc;
    uint32_t cur[kBuckets];
    memcpy(cur, offsets, sizeof cur);
    for (int e = 0; e < n_taps; e++)
        for (int d = 0; d < kDigits; d++) {
            const int v = dig[e][d];
            if (!v) continue;
            items[cur[abs(v) - 1]++] = (uint32_t)e | ((uint32_t)d << 8) | ((v < 0 ? 1u : 0u) << 16);
        }
    if (perm) {
        std::vector<int> order(kBuckets);
        for (int k = 0; k < kBuckets; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return std::min(count[a], 63u) > std::min(count[b], 63u);
        });
        for (int k = 0; k < kBuckets; k++) perm[k] = (uint32_t)order[k];
    }
}

// Phase-B half taps c+-[e] = (c[e] +- c[e+64]) / 2 (one fold), recoded and
// grouped per half; split_phi as in tap_digits.
bool host_tap_tables(const std::vector<Fr> &fwd, std::vector<uint32_t> items[2], uint32_t offsets[2][kBuckets + 1],
                     uint32_t perm[2][kBuckets], bool split_phi) {
    Fr c[kCells];
    host_taps128(fwd, c);
    const Fr inv2 = fr_inv(fr_from_u32(2));
    for (int h = 0; h < 2; h++) {
        int dig[kHalf][kDigits];
        for (int e = 0; e < kHalf; e++) {
            const Fr tap = fr_mul(h == 0 ? fr_add(c[e], c[e + kHalf]) : fr_sub(c[e], c[e + kHalf]), inv2);
            if (!tap_digits(tap, split_phi, dig[e])) return false;
        }
        items[h].assign((size_t)kHalf * kDigits, 0);
        group_items(dig, kHalf, items[h].data(), offsets[h], perm[h]);
        items[h].resize(offsets[h][kBuckets]);
    }
    return true;
}

// Tap items of the parts of `levels` folds (part_layout), split for phi: the
// taps fold like the points, t+-[e] = (t[e] +- t[e + m]) / 2.  items holds
// 32 * 128 entries, part q's from 32 * off[q].  Then, per part, pairs of items
// that share a bucket are replaced by one item on a shared pair sum (DerivType)
// wherever the same pair -- rows, tap distance, relative sign -- occurs twice or
// more (in one bucket or several): greedily, the most frequent pair first, each
// item used once.
// A shared pair sum costs n additions per blob and saves n per extra use.
bool host_part_tables(const std::vector<Fr> &fwd, int levels, std::vector<uint32_t> &items,
                      uint32_t offsets[kFBMaxParts][kBuckets + 1], std::vector<DerivType> &types) {
    const PartLayout L = part_layout(levels);
    Fr v[kCells];
    host_taps128(fwd, v);
    const Fr inv2 = fr_inv(fr_from_u32(2));
    std::vector<Fr> taps[kFBMaxParts];
    for (int l = 1; l <= levels; l++) {
        const int m = kCells >> l;
        std::vector<Fr> &neg = taps[levels + 1 - l];
        neg.resize(m);
        for (int e = 0; e < m; e++) {
            neg[e] = fr_mul(fr_sub(v[e], v[e + m]), inv2);
            v[e] = fr_mul(fr_add(v[e], v[e + m]), inv2);
        }
    }
    taps[0].assign(v, v + (kCells >> levels));
    items.assign((size_t)kCells * kDigits, 0);
    memset(offsets, 0, sizeof(uint32_t) * kFBMaxParts * (kBuckets + 1));
    types.clear();
    struct Item {
        int e, d, neg;
    };
    struct Occ {
        int k, i, j;
    };
    for (int q = 0; q < L.n; q++) {
        const int n = (int)L.size[q];
        std::vector<std::array<int, kDigits>> dig(n);
        for (int e = 0; e < n; e++)
            if (!tap_digits(taps[q][e], true, dig[e].data())) return false;
        std::vector<std::vector<Item>> bk(kBuckets);
        for (int e = 0; e < n; e++)
            for (int d = 0; d < kDigits; d++)
                if (dig[e][d]) bk[abs(dig[e][d]) - 1].push_back({e, d, dig[e][d] < 0 ? 1 : 0});
        // every pair of items in a bucket, keyed by (row a, row b, delta, relative sign)
        std::map<std::array<int, 4>, std::vector<Occ>> occ;
        for (int k = 0; k < kBuckets; k++)
            for (int i = 0; i < (int)bk[k].size(); i++)
                for (int j = i + 1; j < (int)bk[k].size(); j++) {
                    int ia = i, ib = j;
                    const Item &x = bk[k][i], &y = bk[k][j];
                    if (std::make_pair(y.d, y.e) < std::make_pair(x.d, x.e)) std::swap(ia, ib);
                    const Item &A = bk[k][ia], &B = bk[k][ib];
                    int delta = B.e - A.e, sgn = A.neg ^ B.neg;
                    if (delta < 0) {
                        delta += n;
                        if (L.nega[q]) sgn ^= 1; // L~[y - n] = -L~[y]
                    }
                    occ[{A.d, B.d, delta, sgn}].push_back({k, ia, ib});
                }
        std::vector<std::pair<const std::array<int, 4> *, const std::vector<Occ> *>> order;
        for (const auto &kv : occ)
            if (kv.second.size() >= 2) order.push_back({&kv.first, &kv.second});
        std::stable_sort(order.begin(), order.end(),
                         [](const auto &x, const auto &y) { return x.second->size() > y.second->size(); });
        std::vector<std::vector<char>> used(kBuckets);
        for (int k = 0; k < kBuckets; k++) used[k].assign(bk[k].size(), 0);
        std::vector<std::vector<Item>> extra(kBuckets);
        int t = 0;
        for (const auto &ty : order) {
            if (t >= kMaxPartTypes) break;
            std::vector<Occ> sel;
            for (const Occ &o : *ty.second)
                if (!used[o.k][o.i] && !used[o.k][o.j]) {
                    sel.push_back(o);
                    used[o.k][o.i] = used[o.k][o.j] = 1;
                }
            if (sel.size() < 2) {
                for (const Occ &o : sel) used[o.k][o.i] = used[o.k][o.j] = 0;
                continue;
            }
            const std::array<int, 4> &key = *ty.first;
            types.push_back({(uint8_t)q, (uint8_t)key[0], (uint8_t)key[1], (uint8_t)key[3], (uint32_t)key[2], 0});
            for (const Occ &o : sel) extra[o.k].push_back({bk[o.k][o.i].e, kDigits + t, bk[o.k][o.i].neg});
            t++;
        }
        uint32_t *dst = items.data() + (size_t)kDigits * L.off[q];
        uint32_t acc = 0;
        for (int k = 0; k < kBuckets; k++) {
            offsets[q][k] = acc;
            auto put = [&](const Item &it) {
                dst[acc++] = (uint32_t)it.e | ((uint32_t)it.d << 8) | ((uint32_t)it.neg << 16);
            };
            for (size_t i = 0; i < bk[k].size(); i++)
                if (!used[k][i]) put(bk[k][i]);
            for (const Item &it : extra[k]) put(it);
        }
        offsets[q][kBuckets] = acc;
        if (acc > (uint32_t)(kDigits * n)) return false;
    }
    return true;
}

struct HostTables {
    std::vector<uint8_t> pos; // may be empty when generated on the device
    std::vector<Fr> roots_fwd, roots_inv;
    std::vector<uint32_t> items[2];
    uint32_t offsets[2][kBuckets + 1];
    uint32_t perm[2][kBuckets];
    Fr inv_blob;
};

bool read_exact(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

// precomputed_tables.bin, format v1 (src/precomputed_tables.cpp:16-58)
vkzg_result load_tables_file(const char *path, HostTables &h) {
    FILE *f = fopen(path, "rb");
    if (!f) return VKZG_ERR_IO;
    vkzg_result rc = VKZG_ERR_SETUP;
    uint32_t hdr[4];
    // each half holds at most one item per (tap, digit): 64 x 32 (the phase-B
    // kernels size their shared memory and scratch by that bound)
    if (read_exact(f, hdr, 16) && hdr[0] == 0x475A4B56u && hdr[1] == 1u && hdr[2] <= (uint32_t)(kHalf * kDigits) &&
        hdr[3] <= (uint32_t)(kHalf * kDigits)) {
        h.pos.resize(kPositionPoints * sizeof(G1A));
        h.roots_fwd.resize(kExtElems);
        h.roots_inv.resize(kExtElems);
        h.items[0].resize(hdr[2]);
        h.items[1].resize(hdr[3]);
        if (read_exact(f, h.pos.data(), h.pos.size()) && read_exact(f, h.roots_fwd.data(), kExtElems * sizeof(Fr)) &&
            read_exact(f, h.roots_inv.data(), kExtElems * sizeof(Fr)) &&
            read_exact(f, h.items[0].data(), 4 * (size_t)hdr[2]) &&
            read_exact(f, h.items[1].data(), 4 * (size_t)hdr[3]) && read_exact(f, h.offsets[0], sizeof h.offsets[0]) &&
            read_exact(f, h.offsets[1], sizeof h.offsets[1]) && read_exact(f, h.perm[0], sizeof h.perm[0]) &&
            read_exact(f, h.perm[1], sizeof h.perm[1]) && read_exact(f, &h.inv_blob, sizeof h.inv_blob)) {
            rc = VKZG_OK;
            // index sanity: offsets monotone within the item counts, perm a permutation
            for (int s = 0; s < 2 && rc == VKZG_OK; s++) {
                if (h.offsets[s][0] != 0 || h.offsets[s][kBuckets] != hdr[2 + s]) rc = VKZG_ERR_SETUP;
                for (int k = 0; k < kBuckets && rc == VKZG_OK; k++)
                    if (h.offsets[s][k] > h.offsets[s][k + 1] || h.perm[s][k] >= (uint32_t)kBuckets) rc = VKZG_ERR_SETUP;
                for (uint32_t it = 0; it < hdr[2 + s] && rc == VKZG_OK; it++)
                    if ((h.items[s][it] & 0xffu) >= (uint32_t)kHalf || ((h.items[s][it] >> 8) & 0xffu) >= (uint32_t)kDigits)
                        rc = VKZG_ERR_SETUP;
            }
        }
    }
    fclose(f);
    return rc;
}

vkzg_result read_file(const std::string &path, std::vector<uint8_t> &out) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return VKZG_ERR_IO;
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    const bool ok = n > 0 && read_exact(f, out.data(), out.size());
    fclose(f);
    return ok ? VKZG_OK : VKZG_ERR_SETUP;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        if ((call) != cudaSuccess) return VKZG_ERR_GPU;                                               \
    } while (0)

// The device's phase-B tables are always the split ones, computed from the
// roots (a tables file's own items are the reference's 32-digit recoding and
// are kept only for writing the file back out).
vkzg_result upload_small_tables(vkzg_prover *p, const HostTables &h) {
    DeviceTables &t = p->t;
    std::vector<uint32_t> items[2];
    uint32_t offsets[2][kBuckets + 1], perm[2][kBuckets];
    if (!host_tap_tables(h.roots_fwd, items, offsets, perm, true)) return VKZG_ERR_SETUP;
    if (!p->alloc(t.roots_fwd, kExtElems) || !p->alloc(t.roots_inv, kExtElems) || !p->alloc(t.shift_fwd, kExtElems) ||
        !p->alloc(t.shift_inv, kExtElems) || !p->alloc(t.inv_blob_r2, 1))
        return VKZG_ERR_MALLOC;
    for (int s = 0; s < 2; s++) {
        if (!p->alloc(t.tap_items[s], std::max<size_t>(1, items[s].size())) || !p->alloc(t.tap_offsets[s], kBuckets + 1) ||
            !p->alloc(t.tap_perm[s], kBuckets))
            return VKZG_ERR_MALLOC;
        CK(cudaMemcpy(t.tap_items[s], items[s].data(), 4 * items[s].size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(t.tap_offsets[s], offsets[s], sizeof offsets[s], cudaMemcpyHostToDevice));
        CK(cudaMemcpy(t.tap_perm[s], perm[s], sizeof perm[s], cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(t.roots_fwd, h.roots_fwd.data(), kExtElems * sizeof(Fr), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.roots_inv, h.roots_inv.data(), kExtElems * sizeof(Fr), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.inv_blob_r2, &h.inv_blob, sizeof(Fr), cudaMemcpyHostToDevice));
    // plans 3-4: the tap items of the kPartLevels parts and their round structure
    {
        std::vector<uint32_t> pitems;
        uint32_t poffs[kFBMaxParts][kBuckets + 1];
        std::vector<DerivType> types;
        if (!host_part_tables(h.roots_fwd, kPartLevels, pitems, poffs, types)) return VKZG_ERR_SETUP;
        if (!p->alloc(t.part_items, pitems.size()) || !p->alloc(t.part_offsets, (size_t)kFBMaxParts * (kBuckets + 1)))
            return VKZG_ERR_MALLOC;
        CK(cudaMemcpy(t.part_items, pitems.data(), 4 * pitems.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(t.part_offsets, poffs, sizeof poffs, cudaMemcpyHostToDevice));
        // shared pair sums: part q's types follow each other, n_q points each
        const PartLayout PL = part_layout(kPartLevels);
        uint32_t dp = 0;
        for (int q = 0; q < PL.n; q++) {
            t.deriv_base[q] = dp;
            for (auto &ty : types)
                if (ty.part == q) {
                    ty.base = dp;
                    dp += PL.size[q];
                }
        }
        t.deriv_points = dp;
        t.deriv_types = (int)types.size();
        if (dp) {
            std::vector<uint16_t> of(dp);
            for (size_t i = 0; i < types.size(); i++)
                for (uint32_t x = 0; x < PL.size[types[i].part]; x++) of[types[i].base + x] = (uint16_t)i;
            if (!p->alloc(t.deriv, types.size()) || !p->alloc(t.deriv_of, dp)) return VKZG_ERR_MALLOC;
            CK(cudaMemcpy(t.deriv, types.data(), sizeof(DerivType) * types.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(t.deriv_of, of.data(), 2 * (size_t)dp, cudaMemcpyHostToDevice));
        }
        std::unique_ptr<FlatBPlan> pl(new FlatBPlan);
        if (build_flatb_plan(part_layout(kPartLevels), poffs, *pl) && pl->rounds > 0) {
            if (!p->alloc(t.fb_plan, 1)) return VKZG_ERR_MALLOC;
            CK(cudaMemcpy(t.fb_plan, pl.get(), sizeof(FlatBPlan), cudaMemcpyHostToDevice));
            t.fb_rounds = pl->rounds;
            t.fb_stride[0] = pl->stride[1];
            t.fb_stride[1] = pl->rounds > 1 ? pl->stride[2] : 1;
        }
    }
    // recovery coset-shift tables (the reference's k_pow_seq, src/vkzg.cpp:757-774),
    // with 1/8192 folded in and, for the inverse, an extra 1/R (see recover_kernels.cu)
    std::vector<Fr> sf(kExtElems), si(kExtElems);
    const Fr inv_n = fr_inv(fr_from_u32(kExtElems)), seven = fr_from_u32(7), inv7 = fr_inv(seven);
    Fr a = inv_n, b = inv_n;
    for (int k = 0; k < kExtElems; k++) {
        sf[k] = a;
        si[k] = fr_to_canonical(b);
        a = fr_mul(a, seven);
        b = fr_mul(b, inv7);
    }
    CK(cudaMemcpy(t.shift_fwd, sf.data(), kExtElems * sizeof(Fr), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.shift_inv, si.data(), kExtElems * sizeof(Fr), cudaMemcpyHostToDevice));
    return VKZG_OK;
}

// Position table from a setup on the device.
vkzg_result generate_position_table(vkzg_prover *p, const std::vector<uint8_t> &setup) {
    if (setup.size() != (size_t)kBlobElems * 48) return VKZG_ERR_SETUP;
    uint8_t *d_setup = nullptr;
    void *scratch = nullptr;
    uint32_t *d_err = nullptr;
    vkzg_result rc = VKZG_OK;
    if (cudaMalloc(&d_setup, setup.size()) != cudaSuccess || cudaMalloc(&scratch, setup_scratch_bytes()) != cudaSuccess ||
        cudaMalloc(&d_err, 4) != cudaSuccess) {
        rc = VKZG_ERR_MALLOC;
    } else {
        uint32_t h_err = 0;
        if (cudaMemcpy(d_setup, setup.data(), setup.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(d_err, 0, 4) != cudaSuccess ||
            launch_setup_tables(d_setup, p->t.pos, p->t.roots_fwd, scratch, d_err, p->stream) != cudaSuccess ||
            cudaStreamSynchronize(p->stream) != cudaSuccess ||
            cudaMemcpy(&h_err, d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = VKZG_ERR_GPU;
        } else if (h_err) {
            rc = VKZG_ERR_SETUP;
        }
    }
    cudaFree(d_setup);
    cudaFree(scratch);
    cudaFree(d_err);
    return rc;
}

void computed_small_tables(HostTables &h) {
    host_roots(h.roots_fwd, h.roots_inv);
    host_tap_tables(h.roots_fwd, h.items, h.offsets, h.perm, false);
    h.inv_blob = fr_inv(fr_from_u32(kBlobElems));
}

void load_tune_cache(vkzg_prover *p);

vkzg_result alloc_working_set(vkzg_prover *p, uint32_t cap) {
    p->cap = cap;
    ProofWork &w = p->pw;
    RecoverWork &r = p->rw;
    const size_t B = cap;
    bool ok = p->alloc(w.blobs, B * kBlobBytes) && p->alloc(w.coeffs, B * kBlobElems) &&
              p->alloc(w.scalars, B * kCells * kCellElems) && p->alloc(w.buckets, B * kCells * kBuckets) &&
              p->alloc(w.points, B * kCells) && p->alloc(w.ladder, B * kCells * kLadderDigits) &&
              p->alloc(w.ladder_aff, B * kCells * kDigits) &&
              p->alloc(w.proofs, B * kCells * kProofBytes) && p->alloc(w.err, B) &&
              p->alloc(r.cells, B * kExtElems * 32) && p->alloc(r.present, B * kCells) &&
              p->alloc(r.out, B * kExtElems * 32) && p->alloc(r.err, B);
    if (!ok) return VKZG_ERR_MALLOC;
    if (cudaMallocHost(&p->h_err, B * sizeof(uint32_t)) != cudaSuccess) return VKZG_ERR_MALLOC;
    // batch-affine bucket accumulation: one scratch slot per resident block
    // plan override (0 serial Jacobian, 1 batch-affine + binary split, 2 batch-affine + serial)
    if (const char *plan = getenv("VKZG_PLAN")) {
        const int v = atoi(plan);
        if (v >= 0 && v < 5) p->plan_forced = v;
    }
    if (const char *cache = getenv("VKZG_TUNE_CACHE")) p->tune_cache = cache;
    if (const char *g = getenv("VKZG_GRAPHS")) p->use_graphs = atoi(g) != 0;
    load_tune_cache(p);
    // persistent grid of the batch-affine kernels: a block per resident slot,
    // but no more than the capacity's tasks (kWarpOutputs outputs per warp) fill
    const int warps_per_block = VKZG_BA_THREADS / 32;
    const int tasks = (int)((B * kCells + kWarpOutputs - 1) / kWarpOutputs);
    w.ba_blocks = std::min((int)p->sm_count * batch_affine_blocks_per_sm(),
                           (tasks + warps_per_block - 1) / warps_per_block);
    if (!p->alloc(w.bucket_aff, B * kCells * kBuckets) ||
        !p->alloc(w.ba_scratch, (size_t)w.ba_blocks * kBAScratchPoints) ||
        !p->alloc(w.red_scratch, reduce_scratch_points((int)B)) || !p->alloc(w.task_ctr, 2))
        return VKZG_ERR_MALLOC;
    return VKZG_OK;
}

} // namespace

// -------------------------------------------------------------- lifecycle

static vkzg_result write_tables_file(const char *out_path, const HostTables &h, const G1A *d_pos);

static bool create_sides(vkzg_prover *p) {
    for (auto &x : p->side)
        if (cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) != cudaSuccess) return false;
    for (auto &e : p->side_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
    for (auto &e : p->part_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
    return true;
}

// FNV-1a over 8-byte words (plus the tail), as hex: identifies setup tables.
static std::string hash_hex(const uint8_t *d, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        memcpy(&w, d + i, 8);
        h = (h ^ w) * 0x100000001b3ull;
    }
    for (; i < n; i++) h = (h ^ d[i]) * 0x100000001b3ull;
    char buf[24];
    snprintf(buf, sizeof buf, "%016llx", (unsigned long long)h);
    return buf;
}

vkzg_result vkzg_prover_new(vkzg_prover **out, const vkzg_options *opts) {
    if (!out) return VKZG_ERR_BADARGS;
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return VKZG_ERR_GPU;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return VKZG_ERR_GPU;
    // Kernel attributes are per device: set them on the device this prover uses.
    if (configure_proof_kernels() != cudaSuccess || configure_recover_kernels() != cudaSuccess ||
        configure_cells_kernels() != cudaSuccess)
        return VKZG_ERR_GPU;

    vkzg_prover *p = new (std::nothrow) vkzg_prover();
    if (!p) return VKZG_ERR_MALLOC;
    p->device = dev;
    p->name = prop.name;
    p->sm_count = (uint32_t)prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete p;
        return VKZG_ERR_GPU;
    }
    for (auto &e : p->ev_rec)
        if (cudaEventCreate(&e) != cudaSuccess) {
            delete p;
            return VKZG_ERR_GPU;
        }
    for (auto &e : p->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            delete p;
            return VKZG_ERR_GPU;
        }
    if (cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&p->ev_tune[0]) != cudaSuccess || cudaEventCreate(&p->ev_tune[1]) != cudaSuccess ||
        !create_sides(p)) {
        delete p;
        return VKZG_ERR_GPU;
    }

    // Setup tables: file first, in the reference's search order, then device generation.
    const std::string libdir = library_dir();
    std::vector<std::string> files;
    if (const char *env = getenv("VKZG_TABLES_PATH")) files.push_back(env);
    const char *cache = getenv("VKZG_TABLES_CACHE");
    if (cache && *cache) files.push_back(cache);
    files.push_back(libdir + "/precomputed_tables.bin");
    HostTables h;
    vkzg_result rc = VKZG_ERR_IO;
    bool seen_malformed = false;
    for (const auto &f : files) {
        rc = load_tables_file(f.c_str(), h);
        if (rc == VKZG_OK) {
            p->tables_source = "file:" + f;
            p->tables_id = "pos:" + hash_hex(h.pos.data(), h.pos.size());
            break;
        }
        if (rc == VKZG_ERR_SETUP) seen_malformed = true;
    }
    if (rc == VKZG_OK) {
        if (!p->alloc(p->t.pos, kPositionPoints)) rc = VKZG_ERR_MALLOC;
        else if (cudaMemcpy(p->t.pos, h.pos.data(), h.pos.size(), cudaMemcpyHostToDevice) != cudaSuccess) rc = VKZG_ERR_GPU;
        else rc = upload_small_tables(p, h);
    } else {
        const char *envs = getenv("VKZG_SETUP_PATH");
        const std::string setup_path = envs ? std::string(envs) : libdir + "/data/trusted_setup_g1_monomial.bin";
        std::vector<uint8_t> setup;
        rc = read_file(setup_path, setup);
        if (rc == VKZG_OK) {
            computed_small_tables(h);
            rc = upload_small_tables(p, h);
            if (rc == VKZG_OK && !p->alloc(p->t.pos, kPositionPoints)) rc = VKZG_ERR_MALLOC;
            if (rc == VKZG_OK) rc = generate_position_table(p, setup);
            if (rc == VKZG_OK) p->tables_source = "generated:" + setup_path;
            p->tables_id = "setup:" + hash_hex(setup.data(), setup.size());
            // setup cache: the next prover loads the file instead of generating
            if (rc == VKZG_OK && cache && *cache && cudaStreamSynchronize(p->stream) == cudaSuccess &&
                write_tables_file(cache, h, p->t.pos) == VKZG_OK)
                p->tables_source += " (cached to " + std::string(cache) + ")";
        } else if (seen_malformed) {
            rc = VKZG_ERR_SETUP;
        }
    }
    p->tables_bytes = p->dev_bytes;
    if (const char *e = getenv("VKZG_COMB_BUDGET_GB")) p->comb_budget = (uint64_t)(atof(e) * (double)(1ull << 30));
    // 0 = the reference's default of 4 blobs per launch (src/vkzg.cpp:699)
    if (rc == VKZG_OK) rc = alloc_working_set(p, opts && opts->max_batch_size ? opts->max_batch_size : 4);
    if (rc == VKZG_OK && cudaStreamSynchronize(p->stream) != cudaSuccess) rc = VKZG_ERR_GPU;
    if (rc != VKZG_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return VKZG_OK;
}

void vkzg_prover_free(vkzg_prover *p) { delete p; }

// ---------------------------------------------------------------- compute

namespace {

void collect_times(const cudaEvent_t *ev, int stages, double *dst) {
    for (int i = 0; i < stages; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        dst[i] = ms;
    }
}

// ---------------------------------------------------------------- autotuner
// Three plans compute identical bytes (section "plan" in launch_proofs_timed):
// serial Jacobian buckets win for a handful of blobs (more, smaller blocks),
// batch-affine rounds win once a chunk fills the GPU, and which reduction is
// faster depends on the chunk size.  The first chunk of each power-of-two size
// class is timed under every plan on the stream and the fastest is kept.

constexpr int kPlans = 5;

// plan 3's table and buffers, from the prover's working set into a copy of it
void take_comb(ProofWork &w, const ProofWork &from) {
    w.comb = from.comb;
    w.comb_windows = from.comb_windows;
    w.flat_dig = from.flat_dig;
    w.flat_buf[0] = from.flat_buf[0];
    w.flat_buf[1] = from.flat_buf[1];
    w.flat_pre = from.flat_pre;
    w.flat_others = from.flat_others;
    w.flat_tot = from.flat_tot;
    w.flat_totinv = from.flat_totinv;
    w.flat_slots = from.flat_slots;
    w.flat_blocks = from.flat_blocks;
    w.flatb_buf[0] = from.flatb_buf[0];
    w.flatb_buf[1] = from.flatb_buf[1];
    w.deriv_buf = from.deriv_buf;
    w.coop = from.coop;
    w.sync = from.sync;
}

// The proof pipeline of one chunk on the prover's own working set (p->pw with
// w.plan): 10 to ~45 launches, captured once per (chunk size, plan) into a CUDA
// graph and replayed with one cudaGraphLaunch.  Launched directly while stage
// timing is on, for sizes beyond the cache (kMaxGraphs), or when $VKZG_GRAPHS=0.
constexpr size_t kMaxGraphs = 160; // every chunk size of a 128-blob serving lane, and then some

// the captured pipeline of (n, w.plan), captured now if it is not yet; *rec is
// null when graphs are off or the cache is full
// rest_only: the pipeline without stages 1-2 (launched per upload piece)
cudaError_t proof_graph(vkzg_prover *p, const ProofWork &w, uint32_t n, const vkzg_prover::GraphRec **rec,
                        bool rest_only = false) {
    *rec = nullptr;
    const uint64_t key = ((uint64_t)n << 8) | (uint64_t)w.plan | (rest_only ? 0x80u : 0u);
    auto it = p->graphs.find(key);
    if (p->timing || !p->use_graphs || (it == p->graphs.end() && p->graphs.size() >= kMaxGraphs)) return cudaSuccess;
    if (it == p->graphs.end()) {
        cudaStream_t s = p->stream;
        const uint64_t before = t_launches;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        e = launch_proofs_timed(p->t, w, (int)n, s, nullptr, rest_only);
        const cudaError_t e2 = cudaStreamEndCapture(s, &g);
        const uint64_t k = t_launches - before;
        count_launches(-(int)k); // captured, not run
        if (e == cudaSuccess) e = e2;
        cudaGraphExec_t ex = nullptr;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        it = p->graphs.emplace(key, vkzg_prover::GraphRec{ex, k}).first;
    }
    *rec = &it->second;
    return cudaSuccess;
}

cudaError_t run_proofs(vkzg_prover *p, const ProofWork &w, uint32_t n) {
    const vkzg_prover::GraphRec *rec = nullptr;
    const cudaError_t e = proof_graph(p, w, n, &rec);
    if (e != cudaSuccess) return e;
    if (!rec) return launch_proofs_timed(p->t, w, (int)n, p->stream, p->timing ? p->ev : nullptr);
    count_launches((int)rec->launches);
    return cudaGraphLaunch(rec->exec, p->stream);
}
// Size classes below this take the digit table only in a prover whose
// max_batch_size reaches it (it builds the table for its larger chunks anyway),
// at the fewest-window candidate: the window count is chosen at the larger
// classes.  With the table built, plan 3 measured fastest down to one blob
// (3.0 against 4.0 ms for plan 0, 3.7 against 6.2 ms at 8 blobs).
constexpr uint32_t kCombMinBlobs = 16;

// ------------------------------------------------------------ digit table
std::mutex g_comb_mu;
std::map<std::string, std::weak_ptr<CombTable>> g_comb;
// the window a tuner chose, per device, setup tables and budget: later provers
// of the process with the same budget take it (and so share the table)
std::map<std::string, int> g_comb_choice;
std::string comb_choice_key(const vkzg_prover *p) {
    return std::to_string(p->device) + "|" + p->tables_id + "|" + std::to_string(p->comb_budget);
}

// $VKZG_COMB_WINDOWS pins the digit table's windows per scalar (18..32), or
// $VKZG_COMB_BITS its widest window (D = ceil(256 / bits): 8 bits 32 windows,
// 14 bits 19, 15 bits 18); 0 in either disables the table; -1 when neither is
// set.
int comb_windows_forced() {
    if (const char *e = getenv("VKZG_COMB_WINDOWS")) {
        const int d = atoi(e);
        return d <= 0 ? 0 : std::min(kCombMaxWindows, std::max(kCombMinWindows, d));
    }
    if (const char *e = getenv("VKZG_COMB_BITS")) {
        const int c = atoi(e);
        return c <= 0 ? 0 : std::min(kCombMaxWindows, std::max(kCombMinWindows, (256 + c - 1) / c));
    }
    return -1;
}

size_t comb_bytes(int windows) {
    return (size_t)kCells * kCellElems * comb_windows(windows).entries() * kCombEntryBytes;
}

// The grid-wide rounds' shared working set (prefix products, per-lane and
// per-warp products) and phase B's round buffers: plans 3 and 4.
bool ensure_flat_b(vkzg_prover *p) {
    ProofWork &w = p->pw;
    if (w.flat_pre) return true;
    // (chunks beyond 4096 blobs would overflow the rounds' 32-bit pair indices)
    if (p->flat_failed || p->t.fb_rounds == 0 || p->cap > 4096) return false;
    const FlatSizes z = flat_sizes((int)p->cap, kCombMaxWindows); // its slots cover every table and phase B
    if (!p->alloc(w.flat_pre, z.pre_words) || !p->alloc(w.flat_others, z.lanes) ||
        !p->alloc(w.flat_tot, z.lanes / 32) || !p->alloc(w.flat_totinv, z.lanes / 32) ||
        !p->alloc(w.flatb_buf[0], (size_t)p->cap * kCells * std::max<uint32_t>(1, p->t.fb_stride[0])) ||
        !p->alloc(w.flatb_buf[1], (size_t)p->cap * kCells * std::max<uint32_t>(1, p->t.fb_stride[1])) ||
        !p->alloc(w.deriv_buf, (size_t)p->cap * std::max<uint32_t>(1, p->t.deriv_points))) {
        cudaGetLastError();
        w.flat_pre = nullptr;
        p->flat_failed = true;
        return false;
    }
    w.flat_slots = z.slots;
    w.flat_blocks = z.blocks;
    // $VKZG_COOP=1: the rounds of each phase as one cooperative launch (10
    // launches per proof step instead of ~60); measured 3 % slower than the
    // captured graph of separate launches (the round loop's state pushes the
    // passes past 128 registers), so it is not the default
    const char *coop = getenv("VKZG_COOP");
    if (!p->coop_off && coop && atoi(coop) != 0 && coop_supported(z.blocks / (int)p->sm_count) &&
        p->alloc(w.sync, 4))
        w.coop = true;
    cudaGetLastError();
    return true;
}

// Window counts the tuner tries, largest table first: the fewest windows
// whose table fits the prover's budget and the next two (each window more
// adds 64 points to every phase-A output, ~5 %, and shrinks the table by
// about a third), or the pinned or chosen count.
std::vector<int> comb_candidates(const vkzg_prover *p) {
    const int forced = comb_windows_forced();
    if (forced == 0) return {};
    if (forced > 0) return {forced};
    if (p->comb_windows_chosen) return {p->comb_windows_chosen};
    {
        std::lock_guard<std::mutex> lk(g_comb_mu);
        auto it = g_comb_choice.find(comb_choice_key(p));
        if (it != g_comb_choice.end()) return {it->second};
    }
    std::vector<int> out;
    for (int d = kCombMinWindows; d <= kCombMaxWindows && out.size() < 3; d++)
        if (comb_bytes(d) <= p->comb_budget) out.push_back(d);
    return out;
}

// This prover's phase-A round buffers, sized for d_max windows (more windows
// mean longer lists): they then serve every count <= d_max.
bool comb_buffers(vkzg_prover *p, int d_max) {
    if (p->comb_buf_windows) return d_max <= p->comb_buf_windows;
    const FlatSizes z = flat_sizes((int)p->cap, d_max);
    ProofWork &w = p->pw;
    if (!ensure_flat_b(p) || !p->alloc(w.flat_dig, z.dig) || !p->alloc(w.flat_buf[0], z.buf0) ||
        !p->alloc(w.flat_buf[1], z.buf1)) {
        cudaGetLastError();
        w.flat_dig = nullptr;
        return false;
    }
    p->comb_buf_windows = d_max;
    return true;
}

void drop_comb(vkzg_prover *p) {
    p->comb.reset();
    p->pw.comb = nullptr;
    p->pw.comb_windows = 0;
}

// Shares or builds the digit table of d windows (a new one only when it fits
// in free device memory with 4 GB to spare); the prover's previous table, if
// another, is released first.
bool use_comb(vkzg_prover *p, int d) {
    if (p->comb && p->comb->windows == d) return true;
    drop_comb(p);
    if (!comb_buffers(p, d)) return false;
    std::lock_guard<std::mutex> lk(g_comb_mu);
    const std::string key = std::to_string(p->device) + "|" + std::to_string(d) + "|" + p->tables_id;
    auto it = g_comb.find(key);
    if (it != g_comb.end()) p->comb = it->second.lock();
    if (!p->comb) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
        const size_t bytes = comb_bytes(d);
        if (free_b < bytes + comb_build_scratch_bytes(d) + (4ull << 30)) return false;
        auto t = std::make_shared<CombTable>();
        t->device = p->device;
        t->windows = d;
        t->bytes = bytes;
        if (cudaMalloc(&t->d, bytes) != cudaSuccess) {
            t->d = nullptr;
            cudaGetLastError();
            return false;
        }
        void *scratch = nullptr;
        if (cudaMalloc(&scratch, comb_build_scratch_bytes(d)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        const auto t0 = std::chrono::steady_clock::now();
        cudaError_t e = launch_comb_table(p->t, t->d, scratch, d, p->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
        cudaFree(scratch);
        if (e != cudaSuccess) return false;
        t->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        g_comb[key] = t;
        p->comb = t;
    }
    p->pw.comb = p->comb->d;
    p->pw.comb_windows = p->comb->windows;
    return true;
}

// The digit table of the chosen window count, or of the largest candidate that
// can be had (plan 3 outside the tuner: device-pointer calls, adopted tuning).
bool ensure_comb(vkzg_prover *p) {
    if (p->comb) return true;
    if (p->comb_failed) return false;
    const std::vector<int> cands = comb_candidates(p);
    if (!cands.empty() && comb_buffers(p, cands.back()))
        for (int d : cands)
            if (use_comb(p, d)) return true;
    p->comb_failed = true;
    return false;
}

uint32_t size_class(uint32_t n) {
    uint32_t c = 1;
    while (c < n) c <<= 1;
    return c;
}

void save_tune_cache(const vkzg_prover *p) {
    if (p->tune_cache.empty()) return;
    FILE *f = fopen(p->tune_cache.c_str(), "w");
    if (!f) return;
    for (const auto &kv : p->plan_of) fprintf(f, "%s|%u|%u %d\n", p->name.c_str(), p->sm_count, kv.first, kv.second);
    if (p->comb_windows_chosen)
        fprintf(f, "%s|%u|windows %d\n", p->name.c_str(), p->sm_count, p->comb_windows_chosen);
    fclose(f);
}

void load_tune_cache(vkzg_prover *p) {
    if (p->tune_cache.empty()) return;
    FILE *f = fopen(p->tune_cache.c_str(), "r");
    if (!f) return;
    char line[512];
    const std::string key = p->name + "|" + std::to_string(p->sm_count) + "|";
    while (fgets(line, sizeof line, f)) {
        std::string l(line);
        if (l.compare(0, key.size(), key) != 0) continue;
        unsigned c = 0;
        int plan = -1, window = 0;
        if (sscanf(l.c_str() + key.size(), "%u %d", &c, &plan) == 2 && plan >= 0 && plan < kPlans) p->plan_of[c] = plan;
        else if (sscanf(l.c_str() + key.size(), "windows %d", &window) == 1 && window >= kCombMinWindows &&
                 window <= kCombMaxWindows && comb_bytes(window) <= p->comb_budget)
            p->comb_windows_chosen = window;
    }
    fclose(f);
}

// Runs every plan on w (already holding n blobs), keeps the fastest; the
// outputs left in w are those of the last run (identical for all plans).
vkzg_result tune_chunk(vkzg_prover *p, ProofWork w, uint32_t n) {
    cudaStream_t s = p->stream;
    std::array<double, kPlans> ms{};
    auto time_plan = [&](int plan, double &best) -> vkzg_result {
        w.plan = plan;
        take_comb(w, p->pw);
        best = 1e30;
        for (int rep = 0; rep < 2; rep++) { // the first run of a plan also pays its first-launch costs
            CK(cudaEventRecord(p->ev_tune[0], s));
            CK(launch_proofs_timed(p->t, w, (int)n, s, nullptr));
            CK(cudaEventRecord(p->ev_tune[1], s));
            CK(cudaEventSynchronize(p->ev_tune[1]));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, p->ev_tune[0], p->ev_tune[1]));
            best = std::min(best, (double)t);
        }
        return VKZG_OK;
    };
    for (int plan = 0; plan < kPlans; plan++) {
        ms[plan] = 1e30; // not available at this size or in this memory
        if (plan == 4 && !ensure_flat_b(p)) continue;
        if (plan == 3) {
            // the digit table's window count: every candidate timed, its table
            // size the cost (the budget bounds it), the fastest kept
            const bool small = size_class(n) < kCombMinBlobs;
            std::vector<int> cands = small && p->cap < kCombMinBlobs ? std::vector<int>{} : comb_candidates(p);
            if (cands.empty() || !comb_buffers(p, cands.back())) continue;
            if (small) cands.resize(1);
            std::vector<vkzg_prover::WindowTrial> trials;
            int best_d = 0;
            for (int d : cands) {
                if (!use_comb(p, d)) continue;
                double t = 0.0;
                const vkzg_result rc = time_plan(3, t);
                if (rc != VKZG_OK) return rc;
                trials.push_back({d, p->comb->bytes, p->comb->build_ms, t});
                if (t < ms[3]) {
                    ms[3] = t;
                    best_d = d;
                }
            }
            if (!small) p->window_trials[size_class(n)] = trials;
            if (best_d && small) {
                if (!use_comb(p, best_d)) ms[3] = 1e30;
            } else if (best_d) {
                p->comb_windows_chosen = best_d;
                if (comb_windows_forced() < 0) {
                    std::lock_guard<std::mutex> lk(g_comb_mu);
                    g_comb_choice[comb_choice_key(p)] = best_d;
                }
                if (!use_comb(p, best_d)) ms[3] = 1e30;
            }
            continue;
        }
        const vkzg_result rc = time_plan(plan, ms[plan]);
        if (rc != VKZG_OK) return rc;
    }
    const uint32_t c = size_class(n);
    p->plan_ms[c] = ms;
    p->plan_of[c] = (int)(std::min_element(ms.begin(), ms.end()) - ms.begin());
    save_tune_cache(p);
    return VKZG_OK;
}

// Plan for a chunk of n blobs: forced, tuned, or (device-pointer calls that
// cannot stop to measure) a size rule fitted to the B200 measurements.
int planned(const vkzg_prover *p, uint32_t n) {
    if (p->plan_forced >= 0) return p->plan_forced;
    auto it = p->plan_of.find(size_class(n));
    if (it != p->plan_of.end()) return it->second;
    if (p->comb) return 3; // measured fastest at every size once built
    if (n >= 128) return p->pw.flat_pre ? 4 : 1;
    return n >= 8 ? 2 : 0;
}

// planned(), with the digit table or the grid-wide buffers made ready for plans
// 3 and 4 (plan 1 without them)
int plan_for(vkzg_prover *p, uint32_t n) {
    int plan = planned(p, n);
    if (plan == 3 && !ensure_comb(p)) plan = ensure_flat_b(p) ? 4 : 1;
    if (plan == 4 && !ensure_flat_b(p)) plan = 1;
    // a trimmed working set (trim_working_set) holds only the tuned plans'
    // buffers: a plan whose buffers went is replaced by plan 3, which every
    // trimmed prover keeps (its classes above the Jacobian buckets' size run it)
    if (p->trimmed && (((plan == 1 || plan == 2 || plan == 4) && !p->pw.ba_scratch) ||
                       (plan == 0 && n > p->plan0_cap)))
        plan = 3;
    return plan;
}

bool tuned(const vkzg_prover *p, uint32_t n) {
    return p->plan_forced >= 0 || p->plan_of.count(size_class(n)) != 0;
}

// True for page-locked host memory (cudaHostAlloc'd or registered), which the
// DMA engines read and write directly.
bool host_pinned(const void *ptr) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host threads of pageable recovery: one per hardware thread, at most kSides
// (a 64 MB memcpy on a 16-thread host of the B200 pool: 15.7 GB/s on one
// thread, 47 on 8, 77 on 16).
unsigned stage_threads() {
    return std::max(1u, std::min<unsigned>(vkzg_prover::kSides, std::thread::hardware_concurrency()));
}

// The staging buffers, allocated on first use; false when pinned memory is
// not available (the caller then copies from the pageable buffer directly).
bool ensure_stage(vkzg_prover *p) {
    if (p->stage_in) return true;
    const size_t bytes = (size_t)p->cap * kExtElems * 32;
    if (cudaHostAlloc(&p->stage_in, bytes, cudaHostAllocDefault) != cudaSuccess) {
        p->stage_in = nullptr;
        cudaGetLastError();
        return false;
    }
    if (cudaHostAlloc(&p->stage_out, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaFreeHost(p->stage_in);
        p->stage_in = p->stage_out = nullptr;
        cudaGetLastError();
        return false;
    }
    p->stage_bytes = bytes;
    return true;
}

// Host blobs of a tuned chunk of >= 64 blobs go up in kUploadPieces pieces on the side
// streams, and the per-blob front of the pipeline (stages 1-2) runs on each piece
// as it lands, so the upload overlaps that work; the rest replays its own graph.
static bool upload_in_pieces(vkzg_prover *p, uint32_t n) {
    return n >= 64 && p->side[0] && p->use_graphs && !p->timing && tuned(p, n);
}

// Pageable blobs into the proof working set through the pinned staging: parts
// of kRecPartBlobs blobs or more dealt to host threads (half the hardware
// threads, at most 8; parts t, t + T, ... to thread t, on side stream t), each
// part copied into the staging and its copy up enqueued at once, so that the
// DMA of the first parts runs while later parts are still being copied on the
// host (all 16 hardware threads, copying 2 MB pieces, made the 256-blob call
// 0.5 ms slower than 8).  The copies start after the prover stream's earlier work (which may
// still read the blobs).  On return every copy is enqueued, part k (blobs
// [k part, (k + 1) part)) is up when p->part_ev[k] is, and *part is the part
// size in blobs.
vkzg_result staged_upload(vkzg_prover *p, const uint8_t *blobs, uint32_t n, uint32_t *part_out) {
    const uint32_t parts = std::max<uint32_t>(1, std::min<uint32_t>(vkzg_prover::kRecMaxParts, n / vkzg_prover::kRecPartBlobs));
    const uint32_t part = (n + parts - 1) / parts;
    const uint32_t used = (n + part - 1) / part;
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const uint32_t T = std::min<uint32_t>(used, std::min(8u, hw / 2));
    CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], p->stream));
    for (uint32_t t = 0; t < T; t++) CK(cudaStreamWaitEvent(p->side[t], p->side_ev[vkzg_prover::kSides], 0));
    auto run_thread = [&](uint32_t t) -> vkzg_result {
        if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
        for (uint32_t k = t; k < used; k += T) {
            const size_t off = (size_t)k * part * kBlobBytes, bytes = (size_t)std::min(part, n - k * part) * kBlobBytes;
            memcpy(p->stage_in + off, blobs + off, bytes);
            CK(cudaMemcpyAsync(p->pw.blobs + off, p->stage_in + off, bytes, cudaMemcpyHostToDevice, p->side[t]));
            CK(cudaEventRecord(p->part_ev[k], p->side[t]));
        }
        return VKZG_OK;
    };
    std::vector<vkzg_result> rcs(T, VKZG_OK);
    std::vector<std::thread> ts;
    for (uint32_t t = 1; t < T; t++) ts.emplace_back([&, t] { rcs[t] = run_thread(t); });
    rcs[0] = run_thread(0);
    for (auto &t : ts) t.join();
    for (vkzg_result rc : rcs)
        if (rc != VKZG_OK) return rc;
    *part_out = part;
    return VKZG_OK;
}

// The prover stream waits for every part of a staged_upload of n blobs.
cudaError_t wait_staged(vkzg_prover *p, uint32_t n, uint32_t part) {
    for (uint32_t k = 0; k * part < n; k++) {
        const cudaError_t e = cudaStreamWaitEvent(p->stream, p->part_ev[k], 0);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Device results (n items of `item` bytes at src) into a caller's pageable
// buffer through the pinned output staging: parts of kRecPartBlobs items or
// more dealt to host threads (one per hardware thread, at most kSides; parts t,
// t + T, ... on side stream t), each thread enqueueing its parts' copies down
// at once and copying each part out on the host as soon as it lands, so that
// the host copies overlap the DMA of later parts.  The copies start after the
// prover stream's earlier work.
vkzg_result staged_download(vkzg_prover *p, uint8_t *dst, const uint8_t *src, uint32_t n, size_t item) {
    const uint32_t parts = std::max<uint32_t>(1, std::min<uint32_t>(vkzg_prover::kRecMaxParts, n / vkzg_prover::kRecPartBlobs));
    const uint32_t part = (n + parts - 1) / parts;
    const uint32_t used = (n + part - 1) / part;
    const uint32_t T = std::min<uint32_t>(used, stage_threads());
    CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], p->stream));
    for (uint32_t t = 0; t < T; t++) CK(cudaStreamWaitEvent(p->side[t], p->side_ev[vkzg_prover::kSides], 0));
    auto run_thread = [&](uint32_t t) -> vkzg_result {
        if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
        for (uint32_t k = t; k < used; k += T) {
            const size_t off = (size_t)k * part * item, bytes = (size_t)std::min(part, n - k * part) * item;
            CK(cudaMemcpyAsync(p->stage_out + off, src + off, bytes, cudaMemcpyDeviceToHost, p->side[t]));
            CK(cudaEventRecord(p->part_ev[k], p->side[t]));
        }
        for (uint32_t k = t; k < used; k += T) {
            const size_t off = (size_t)k * part * item, bytes = (size_t)std::min(part, n - k * part) * item;
            CK(cudaEventSynchronize(p->part_ev[k]));
            memcpy(dst + off, p->stage_out + off, bytes);
        }
        return VKZG_OK;
    };
    std::vector<vkzg_result> rcs(T, VKZG_OK);
    std::vector<std::thread> ts;
    for (uint32_t t = 1; t < T; t++) ts.emplace_back([&, t] { rcs[t] = run_thread(t); });
    rcs[0] = run_thread(0);
    for (auto &t : ts) t.join();
    for (vkzg_result rc : rcs)
        if (rc != VKZG_OK) return rc;
    return VKZG_OK;
}

vkzg_result proofs_chunk(vkzg_prover *p, uint8_t *proofs, const uint8_t *blobs, uint32_t n) {
    cudaStream_t s = p->stream;
    // pageable blobs: through the pinned staging buffer in parts (staged_upload)
    const bool staged = n >= 16 && !host_pinned(blobs) && ensure_stage(p);
    uint32_t spart = 0;
    // the prover stream waits for the staged parts holding blobs [from, to)
    auto wait_parts = [&](uint32_t from, uint32_t to) -> cudaError_t {
        for (uint32_t k = from / spart; k * spart < to; k++) {
            const cudaError_t e = cudaStreamWaitEvent(s, p->part_ev[k], 0);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    if (upload_in_pieces(p, n)) {
        p->pw.plan = plan_for(p, n);
        const vkzg_prover::GraphRec *rec = nullptr;
        CK(proof_graph(p, p->pw, n, &rec, true));
        if (staged) {
            const vkzg_result rc = staged_upload(p, blobs, n, &spart);
            if (rc != VKZG_OK) return rc;
        }
        CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
        // the pieces' copies start after the stream's earlier work (which may still read the blobs)
        if (!staged) CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], s));
        const uint32_t part = (n + vkzg_prover::kUploadPieces - 1) / vkzg_prover::kUploadPieces;
        for (uint32_t off = 0, k = 0; off < n; off += part, k++) {
            const uint32_t cnt = std::min(part, n - off);
            if (staged) {
                CK(wait_parts(off, off + cnt));
            } else {
                CK(cudaStreamWaitEvent(p->side[k], p->side_ev[vkzg_prover::kSides], 0));
                CK(cudaMemcpyAsync(p->pw.blobs + (size_t)off * kBlobBytes, blobs + (size_t)off * kBlobBytes,
                                   (size_t)cnt * kBlobBytes, cudaMemcpyHostToDevice, p->side[k]));
                CK(cudaEventRecord(p->side_ev[k], p->side[k]));
                CK(cudaStreamWaitEvent(s, p->side_ev[k], 0));
            }
            CK(launch_proofs_front(p->t, p->pw, (int)off, (int)cnt, s));
        }
        if (rec) {
            count_launches((int)rec->launches);
            CK(cudaGraphLaunch(rec->exec, s));
        } else {
            CK(launch_proofs_timed(p->t, p->pw, (int)n, s, nullptr, true));
        }
    } else {
        if (staged) {
            const vkzg_result rc = staged_upload(p, blobs, n, &spart);
            if (rc != VKZG_OK) return rc;
            CK(wait_staged(p, n, spart));
        } else {
            CK(cudaMemcpyAsync(p->pw.blobs, blobs, (size_t)n * kBlobBytes, cudaMemcpyHostToDevice, s));
        }
        CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
        if (!tuned(p, n)) {
            const vkzg_result rc = tune_chunk(p, p->pw, n);
            if (rc != VKZG_OK) return rc;
        }
        p->pw.plan = plan_for(p, n);
        CK(run_proofs(p, p->pw, n));
    }
    CK(cudaMemcpyAsync(p->h_err, p->pw.err, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (p->timing) collect_times(p->ev, kProofStages, p->last_proof_ms);
    for (uint32_t b = 0; b < n; b++)
        if (p->h_err[b] & kSyncFailed) return VKZG_ERR_GPU;
    for (uint32_t b = 0; b < n; b++)
        if (p->h_err[b]) return VKZG_ERR_INVALID_BLOB;
    CK(cudaMemcpyAsync(proofs, p->pw.proofs, (size_t)n * kCells * kProofBytes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return VKZG_OK;
}

vkzg_result recover_chunk(vkzg_prover *p, uint8_t *out, const uint8_t *cells, const uint8_t *present, uint32_t n) {
    // more than 64 missing cells in any blob of the chunk: BADARGS before any
    // device work for it (src/vkzg.cpp:1093-1105)
    for (uint32_t b = 0; b < n; b++) {
        int miss = 0;
        for (int i = 0; i < kCells; i++) miss += present[(size_t)b * kCells + i] == 0;
        if (miss > kCellElems) return VKZG_ERR_BADARGS;
    }
    cudaStream_t s = p->stream;
    const size_t ext = (size_t)kExtElems * 32;
    const bool pin_in = host_pinned(cells), pin_out = host_pinned(out);
    if (!p->timing && n >= 16 && p->side[0] && (!pin_in || !pin_out) && ensure_stage(p)) {
        // pageable cells or output: parts of at least kRecPartBlobs blobs
        // through the pinned staging buffers, dealt to host threads (parts t,
        // t + T, ... to thread t, each thread on its own side stream).  A thread
        // copies each of its parts in and enqueues the part's copy in, kernel
        // and copy out, then waits for its parts in turn and copies each out, so
        // that its host copies overlap the DMA and kernels of its other parts
        // and of the other threads' parts.
        const uint32_t parts = std::min<uint32_t>(vkzg_prover::kRecMaxParts, n / vkzg_prover::kRecPartBlobs);
        const uint32_t part = (n + parts - 1) / parts;
        const uint32_t used = (n + part - 1) / part;
        const uint32_t T = std::min<uint32_t>(used, stage_threads());
        CK(cudaMemcpyAsync(p->rw.present, present, (size_t)n * kCells, cudaMemcpyHostToDevice, s));
        CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], s));
        for (uint32_t t = 0; t < T; t++) CK(cudaStreamWaitEvent(p->side[t], p->side_ev[vkzg_prover::kSides], 0));
        auto run_thread = [&](uint32_t t) -> vkzg_result {
            if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
            cudaStream_t st = p->side[t];
            for (uint32_t k = t; k < used; k += T) {
                const uint32_t off = k * part, cnt = std::min(part, n - off);
                RecoverWork w = p->rw;
                w.cells += off * ext;
                w.present += (size_t)off * kCells;
                w.out += off * ext;
                w.err += off;
                const uint8_t *src = cells + off * ext;
                if (!pin_in) {
                    memcpy(p->stage_in + off * ext, src, cnt * ext);
                    src = p->stage_in + off * ext;
                }
                CK(cudaMemcpyAsync(w.cells, src, cnt * ext, cudaMemcpyHostToDevice, st));
                CK(launch_recover_timed(p->t, w, (int)cnt, st, nullptr));
                CK(cudaMemcpyAsync(pin_out ? out + off * ext : p->stage_out + off * ext, w.out, cnt * ext,
                                   cudaMemcpyDeviceToHost, st));
                CK(cudaEventRecord(p->part_ev[k], st));
            }
            for (uint32_t k = t; k < used; k += T) {
                const uint32_t off = k * part, cnt = std::min(part, n - off);
                CK(cudaEventSynchronize(p->part_ev[k]));
                if (!pin_out) memcpy(out + off * ext, p->stage_out + off * ext, cnt * ext);
            }
            return VKZG_OK;
        };
        std::vector<vkzg_result> rcs(T, VKZG_OK);
        std::vector<std::thread> ts;
        for (uint32_t t = 1; t < T; t++) ts.emplace_back([&, t] { rcs[t] = run_thread(t); });
        rcs[0] = run_thread(0);
        for (auto &t : ts) t.join();
        for (vkzg_result rc : rcs)
            if (rc != VKZG_OK) return rc;
        return VKZG_OK;
    }
    const uint32_t parts = std::min<uint32_t>(vkzg_prover::kRecMaxParts, n / vkzg_prover::kRecPartBlobs);
    const uint32_t part = n >= vkzg_prover::kPartsFrom && p->side[0] ? (n + parts - 1) / parts : n;
    if (p->timing || part == n) {
        CK(cudaMemcpyAsync(p->rw.cells, cells, n * ext, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(p->rw.present, present, (size_t)n * kCells, cudaMemcpyHostToDevice, s));
        CK(launch_recover_timed(p->t, p->rw, (int)n, s, p->timing ? p->ev_rec : nullptr));
        CK(cudaMemcpyAsync(out, p->rw.out, n * ext, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (p->timing) collect_times(p->ev_rec, kRecoverStages, p->last_recover_ms);
        return VKZG_OK;
    }
    // parts of the chunk on the side streams (after all earlier work of the
    // prover's stream, and after one copy of every blob's presence mask, so
    // that the copy engine's queue holds only the parts' cells)
    CK(cudaMemcpyAsync(p->rw.present, present, (size_t)n * kCells, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], s));
    for (int k = 0; k < vkzg_prover::kSides; k++) CK(cudaStreamWaitEvent(p->side[k], p->side_ev[vkzg_prover::kSides], 0));
    for (uint32_t off = 0, k = 0; off < n; off += part, k++) {
        const uint32_t cnt = std::min(part, n - off);
        cudaStream_t st = p->side[k % vkzg_prover::kSides];
        RecoverWork w = p->rw;
        w.cells += off * ext;
        w.present += (size_t)off * kCells;
        w.out += off * ext;
        w.err += off;
        CK(cudaMemcpyAsync(w.cells, cells + off * ext, cnt * ext, cudaMemcpyHostToDevice, st));
        CK(launch_recover_timed(p->t, w, (int)cnt, st, nullptr));
        CK(cudaMemcpyAsync(out + off * ext, w.out, cnt * ext, cudaMemcpyDeviceToHost, st));
    }
    for (int k = 0; k < vkzg_prover::kSides; k++) {
        CK(cudaEventRecord(p->side_ev[k], p->side[k]));
        CK(cudaStreamWaitEvent(s, p->side_ev[k], 0));
    }
    CK(cudaStreamSynchronize(s));
    return VKZG_OK;
}

} // namespace

vkzg_result vkzg_compute_proofs_batch(vkzg_prover *p, uint8_t *proofs, const uint8_t *blobs, size_t num_blobs) {
    if (!p || !blobs || !proofs) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        const vkzg_result rc = proofs_chunk(p, proofs + done * kCells * kProofBytes, blobs + done * kBlobBytes, n);
        if (rc != VKZG_OK) return rc;
        done += n;
    }
    return VKZG_OK;
}

vkzg_result vkzg_recover_cells_batch(vkzg_prover *p, uint8_t *cells_out, const uint8_t *cells,
                                     const uint8_t *cell_present, size_t num_blobs) {
    if (!p || !cells_out || !cells || !cell_present) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    const size_t blob_bytes = (size_t)kExtElems * 32;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        const vkzg_result rc = recover_chunk(p, cells_out + done * blob_bytes, cells + done * blob_bytes,
                                             cell_present + done * kCells, n);
        if (rc != VKZG_OK) return rc;
        done += n;
    }
    return VKZG_OK;
}

// ------------------------------------------------------------- extensions

void vkzg_b200_set_stage_timing(vkzg_prover *p, int enabled) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mutex);
    p->timing = enabled != 0;
}

int vkzg_b200_last_stage_times(const vkzg_prover *p, int recovery, double *ms, int cap) {
    if (!p || !ms) return 0;
    if (p->pending_proof && cudaEventQuery(p->ev[kProofStages]) == cudaSuccess) {
        collect_times(p->ev, kProofStages, p->last_proof_ms);
        p->pending_proof = false;
    }
    if (p->pending_recover && cudaEventQuery(p->ev_rec[kRecoverStages]) == cudaSuccess) {
        collect_times(p->ev_rec, kRecoverStages, p->last_recover_ms);
        p->pending_recover = false;
    }
    const int n = recovery ? kRecoverStages : kProofStages;
    const double *src = recovery ? p->last_recover_ms : p->last_proof_ms;
    for (int i = 0; i < n && i < cap; i++) ms[i] = src[i];
    return n;
}

const char *vkzg_b200_stage_name(int recovery, int i) {
    if (recovery) return (i >= 0 && i < kRecoverStages) ? kRecoverStageNames[i] : "";
    return (i >= 0 && i < kProofStages) ? kProofStageNames[i] : "";
}

// Writes the tables in the reference's file format (src/precomputed_tables.cpp:
// 16-58): header, position table, roots, phase-B items, offsets, perms,
// 1/4096.  Written to a temporary name and renamed, so a reader never sees a
// partial file.
static vkzg_result write_tables_file(const char *out_path, const HostTables &h, const G1A *d_pos) {
    std::vector<uint8_t> pos(kPositionPoints * sizeof(G1A));
    if (cudaMemcpy(pos.data(), d_pos, pos.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return VKZG_ERR_GPU;
    const std::string tmp_path = std::string(out_path) + ".tmp";
    FILE *f = fopen(tmp_path.c_str(), "wb");
    if (!f) return VKZG_ERR_IO;
    const uint32_t hdr[4] = {0x475A4B56u, 1u, (uint32_t)h.items[0].size(), (uint32_t)h.items[1].size()};
    bool ok = fwrite(hdr, 1, 16, f) == 16 && fwrite(pos.data(), 1, pos.size(), f) == pos.size() &&
              fwrite(h.roots_fwd.data(), sizeof(Fr), kExtElems, f) == (size_t)kExtElems &&
              fwrite(h.roots_inv.data(), sizeof(Fr), kExtElems, f) == (size_t)kExtElems &&
              fwrite(h.items[0].data(), 4, h.items[0].size(), f) == h.items[0].size() &&
              fwrite(h.items[1].data(), 4, h.items[1].size(), f) == h.items[1].size() &&
              fwrite(h.offsets[0], 1, sizeof h.offsets[0], f) == sizeof h.offsets[0] &&
              fwrite(h.offsets[1], 1, sizeof h.offsets[1], f) == sizeof h.offsets[1] &&
              fwrite(h.perm[0], 1, sizeof h.perm[0], f) == sizeof h.perm[0] &&
              fwrite(h.perm[1], 1, sizeof h.perm[1], f) == sizeof h.perm[1] &&
              fwrite(&h.inv_blob, 1, sizeof h.inv_blob, f) == sizeof h.inv_blob;
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp_path.c_str(), out_path) != 0) {
        remove(tmp_path.c_str());
        return VKZG_ERR_IO;
    }
    return VKZG_OK;
}

vkzg_result vkzg_b200_write_tables(const uint8_t *g1_monomial_compressed, const char *out_path) {
    if (!g1_monomial_compressed || !out_path) return VKZG_ERR_BADARGS;
    vkzg_prover tmp; // table storage and stream only
    if (cudaGetDevice(&tmp.device) != cudaSuccess) return VKZG_ERR_GPU;
    if (cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking) != cudaSuccess) return VKZG_ERR_GPU;
    HostTables h;
    computed_small_tables(h);
    vkzg_result rc = upload_small_tables(&tmp, h);
    if (rc == VKZG_OK && !tmp.alloc(tmp.t.pos, kPositionPoints)) rc = VKZG_ERR_MALLOC;
    if (rc != VKZG_OK) return rc;
    std::vector<uint8_t> setup(g1_monomial_compressed, g1_monomial_compressed + (size_t)kBlobElems * 48);
    rc = generate_position_table(&tmp, setup);
    if (rc != VKZG_OK) return rc;
    return write_tables_file(out_path, h, tmp.t.pos);
}

// ------------------------------------------------- device-pointer entry points

namespace {

// caller stream -> prover stream -> caller stream
vkzg_result enter_stream(vkzg_prover *p, cudaStream_t caller) {
    CK(cudaEventRecord(p->ev_in, caller));
    CK(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
    return VKZG_OK;
}
vkzg_result leave_stream(vkzg_prover *p, cudaStream_t caller) {
    CK(cudaEventRecord(p->ev_out, p->stream));
    CK(cudaStreamWaitEvent(caller, p->ev_out, 0));
    return VKZG_OK;
}

} // namespace

vkzg_result vkzg_b200_compute_proofs_device(vkzg_prover *p, uint8_t *d_proofs, const uint8_t *d_blobs,
                                            uint32_t *d_err, size_t num_blobs, void *stream) {
    if (!p || !d_proofs || !d_blobs || !d_err) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    cudaStream_t caller = (cudaStream_t)stream;
    vkzg_result rc = enter_stream(p, caller);
    if (rc != VKZG_OK) return rc;
    // through the working set (two device copies, ~1 % of the chunk's time), so
    // that the pipeline captured for this chunk size replays unchanged
    cudaStream_t s = p->stream;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        CK(cudaMemcpyAsync(p->pw.blobs, d_blobs + done * kBlobBytes, (size_t)n * kBlobBytes, cudaMemcpyDeviceToDevice,
                           s));
        CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
        p->pw.plan = plan_for(p, n);
        CK(run_proofs(p, p->pw, n));
        CK(cudaMemcpyAsync(d_proofs + done * kCells * kProofBytes, p->pw.proofs, (size_t)n * kCells * kProofBytes,
                           cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(d_err + done, p->pw.err, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        done += n;
    }
    if (p->timing) p->pending_proof = true;
    return leave_stream(p, caller);
}

vkzg_result vkzg_b200_recover_cells_device(vkzg_prover *p, uint8_t *d_cells_out, const uint8_t *d_cells,
                                           const uint8_t *d_cell_present, uint32_t *d_err, size_t num_blobs,
                                           void *stream) {
    if (!p || !d_cells_out || !d_cells || !d_cell_present || !d_err) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    cudaStream_t caller = (cudaStream_t)stream;
    vkzg_result rc = enter_stream(p, caller);
    if (rc != VKZG_OK) return rc;
    const size_t blob_bytes = (size_t)kExtElems * 32;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        RecoverWork w = p->rw;
        w.cells = const_cast<uint8_t *>(d_cells) + done * blob_bytes;
        w.present = const_cast<uint8_t *>(d_cell_present) + done * kCells;
        w.out = d_cells_out + done * blob_bytes;
        w.err = d_err + done;
        CK(launch_recover_timed(p->t, w, (int)n, p->stream, p->timing ? p->ev_rec : nullptr));
        done += n;
    }
    if (p->timing) p->pending_recover = true;
    return leave_stream(p, caller);
}

// ------------------------------------------------ allocation-free recovery

namespace vkzg {
int noalloc_max_blobs();
cudaError_t launch_recover_noalloc(const DeviceTables &t, const uint8_t *cells, const uint8_t *present, uint8_t *out,
                                   uint32_t *err, int n, cudaStream_t s);
} // namespace vkzg

vkzg_result vkzg_b200_recover_cells_device_noalloc(vkzg_prover *p, uint8_t *d_cells_out, const uint8_t *d_cells,
                                                   const uint8_t *d_cell_present, uint32_t *d_err,
                                                   size_t num_blobs, void *stream) {
    if (!p || !d_cells_out || !d_cells || !d_cell_present || !d_err) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    if (num_blobs > (size_t)noalloc_max_blobs()) return VKZG_ERR_BADARGS;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return VKZG_ERR_GPU;
    if (dev != p->device) return VKZG_ERR_BADARGS;
    if (launch_recover_noalloc(p->t, d_cells, d_cell_present, d_cells_out, d_err, (int)num_blobs,
                               (cudaStream_t)stream) != cudaSuccess)
        return VKZG_ERR_GPU;
    return VKZG_OK;
}

// ------------------------------------------------- cells (2x RS extension)

namespace vkzg {
cudaError_t launch_cells(const DeviceTables &t, const uint8_t *blobs, uint8_t *cells, uint32_t *err, int n,
                         cudaStream_t s);
} // namespace vkzg

namespace {

// One chunk of compute_cells / compute_cells_and_kzg_proofs: one upload, both
// pipelines on the same device copy of the blobs, outputs written only when
// every blob of the chunk is canonical (the proofs path's rule).
vkzg_result cells_chunk(vkzg_prover *p, uint8_t *cells, uint8_t *proofs, const uint8_t *blobs, uint32_t n) {
    cudaStream_t s = p->stream;
    const size_t ext = (size_t)kExtElems * 32;
    if (!proofs && !p->timing && n >= vkzg_prover::kPartsFrom && p->side[0] && host_pinned(blobs) && host_pinned(cells)) {
        // cells only, page-locked buffers: parts of the chunk on the side
        // streams as recovery runs them (copy in, kernel, copy out per part), so
        // that the 384 KB per blob of copies overlap the kernels.  The cells go
        // out before the blobs' error words are read, so a chunk with an invalid
        // blob has its cells zeroed before INVALID_BLOB is returned.
        const uint32_t parts = std::min<uint32_t>(vkzg_prover::kRecMaxParts, n / vkzg_prover::kRecPartBlobs);
        const uint32_t part = (n + parts - 1) / parts;
        CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
        CK(cudaEventRecord(p->side_ev[vkzg_prover::kSides], s));
        for (int k = 0; k < vkzg_prover::kSides; k++)
            CK(cudaStreamWaitEvent(p->side[k], p->side_ev[vkzg_prover::kSides], 0));
        for (uint32_t off = 0, k = 0; off < n; off += part, k++) {
            const uint32_t cnt = std::min(part, n - off);
            cudaStream_t st = p->side[k % vkzg_prover::kSides];
            CK(cudaMemcpyAsync(p->pw.blobs + (size_t)off * kBlobBytes, blobs + (size_t)off * kBlobBytes,
                               (size_t)cnt * kBlobBytes, cudaMemcpyHostToDevice, st));
            CK(launch_cells(p->t, p->pw.blobs + (size_t)off * kBlobBytes, p->rw.out + off * ext, p->pw.err + off,
                            (int)cnt, st));
            CK(cudaMemcpyAsync(cells + off * ext, p->rw.out + off * ext, cnt * ext, cudaMemcpyDeviceToHost, st));
        }
        for (int k = 0; k < vkzg_prover::kSides; k++) {
            CK(cudaEventRecord(p->side_ev[k], p->side[k]));
            CK(cudaStreamWaitEvent(s, p->side_ev[k], 0));
        }
        CK(cudaMemcpyAsync(p->h_err, p->pw.err, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        vkzg_result rc = VKZG_OK;
        for (uint32_t b = 0; b < n && rc == VKZG_OK; b++)
            if (p->h_err[b] & kSyncFailed) rc = VKZG_ERR_GPU;
        for (uint32_t b = 0; b < n && rc == VKZG_OK; b++)
            if (p->h_err[b]) rc = VKZG_ERR_INVALID_BLOB;
        if (rc != VKZG_OK) memset(cells, 0, (size_t)n * ext);
        return rc;
    }
    // pageable blobs or cells (16 blobs or more): through the pinned staging in
    // parts on host threads (staged_upload, staged_download; 256 blobs of cells
    // from and into pageable buffers 5.4 -> 4.2 ms.  Running each part's upload,
    // kernel and download on the side streams instead, the cells copied out after
    // the error check, measured 4.5-4.8 ms: the per-part launches cost more than
    // the overlap gave)
    const bool stage_blobs = n >= 16 && p->side[0] && !host_pinned(blobs) && ensure_stage(p);
    const bool stage_cells = n >= 16 && p->side[0] && !host_pinned(cells) && ensure_stage(p);
    if (stage_blobs) {
        uint32_t spart = 0;
        const vkzg_result rc = staged_upload(p, blobs, n, &spart);
        if (rc != VKZG_OK) return rc;
        CK(wait_staged(p, n, spart));
    } else {
        CK(cudaMemcpyAsync(p->pw.blobs, blobs, (size_t)n * kBlobBytes, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
    CK(launch_cells(p->t, p->pw.blobs, p->rw.out, p->pw.err, (int)n, s));
    p->pw.plan = plan_for(p, n);
    if (proofs) CK(run_proofs(p, p->pw, n));
    CK(cudaMemcpyAsync(p->h_err, p->pw.err, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (uint32_t b = 0; b < n; b++)
        if (p->h_err[b] & kSyncFailed) return VKZG_ERR_GPU;
    for (uint32_t b = 0; b < n; b++)
        if (p->h_err[b]) return VKZG_ERR_INVALID_BLOB;
    if (proofs) CK(cudaMemcpyAsync(proofs, p->pw.proofs, (size_t)n * kCells * kProofBytes, cudaMemcpyDeviceToHost, s));
    if (stage_cells) {
        const vkzg_result rc = staged_download(p, cells, p->rw.out, n, ext);
        if (rc != VKZG_OK) return rc;
    } else {
        CK(cudaMemcpyAsync(cells, p->rw.out, (size_t)n * ext, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return VKZG_OK;
}

vkzg_result cells_batch(vkzg_prover *p, uint8_t *cells, uint8_t *proofs, const uint8_t *blobs, size_t num_blobs) {
    if (!p || !cells || !blobs) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        const vkzg_result rc = cells_chunk(p, cells + done * (size_t)kExtElems * 32,
                                           proofs ? proofs + done * kCells * kProofBytes : nullptr,
                                           blobs + done * kBlobBytes, n);
        if (rc != VKZG_OK) return rc;
        done += n;
    }
    return VKZG_OK;
}

} // namespace

vkzg_result vkzg_b200_compute_cells_batch(vkzg_prover *p, uint8_t *cells, const uint8_t *blobs, size_t num_blobs) {
    return cells_batch(p, cells, nullptr, blobs, num_blobs);
}

vkzg_result vkzg_b200_compute_cells_and_proofs_batch(vkzg_prover *p, uint8_t *cells, uint8_t *proofs,
                                                     const uint8_t *blobs, size_t num_blobs) {
    if (!proofs) return VKZG_ERR_BADARGS;
    return cells_batch(p, cells, proofs, blobs, num_blobs);
}

// ------------------------------------------------------------ autotuner API

vkzg_result vkzg_b200_autotune(vkzg_prover *p, uint32_t max_blobs) {
    if (!p) return VKZG_ERR_BADARGS;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    const uint32_t top = std::min<uint32_t>(max_blobs ? max_blobs : p->cap, p->cap);
    // size classes from the largest down, so that the digit table's window is
    // chosen at the largest chunk (later classes keep it)
    std::vector<uint32_t> sizes;
    for (uint32_t n = 1; n <= top; n <<= 1) {
        sizes.push_back(n);
        if (n < top && (n << 1) > top) sizes.push_back(top); // finish with the capacity itself
    }
    // seeded canonical blobs (top byte below r's 0x73)
    std::vector<uint8_t> blobs((size_t)top * kBlobBytes);
    uint64_t x = 0x7594ull;
    for (size_t i = 0; i < blobs.size(); i++) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        blobs[i] = (uint8_t)(x >> 24);
        if (i % 32 == 0) blobs[i] &= 0x3f;
    }
    CK(cudaMemcpyAsync(p->pw.blobs, blobs.data(), blobs.size(), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemsetAsync(p->pw.err, 0, top * sizeof(uint32_t), p->stream));
    for (auto it = sizes.rbegin(); it != sizes.rend() && p->plan_forced < 0; ++it) {
        const vkzg_result rc = tune_chunk(p, p->pw, *it);
        if (rc != VKZG_OK) return rc;
    }
    return VKZG_OK;
}

namespace vkzg {
// dst takes src's tuned plans (provers of one serving loop share their
// decisions) and allocates what those plans need now, so that no later call
// stops for a device allocation
// Captures the pipeline of every chunk size 1..max_n (with its tuned plan)
// ahead of use, so that no call waits for a capture (a serving lane meets
// every batch size up to its maximum).
void precapture_graphs(vkzg_prover *p, uint32_t max_n) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return;
    for (uint32_t n = 1; n <= std::min(max_n, p->cap); n++) {
        ProofWork w = p->pw;
        w.plan = plan_for(p, n);
        const vkzg_prover::GraphRec *rec = nullptr;
        if (proof_graph(p, w, n, &rec) != cudaSuccess || !rec) return;
    }
}

void disable_coop(vkzg_prover *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mutex);
    p->coop_off = true;
    p->pw.coop = false;
}

// Frees the buffers that none of the prover's tuned plans uses, so that its
// working set per blob (a serving lane's admission charge) covers only them:
// the per-warp batch-affine scratch when no size class runs plan 1, 2 or 4,
// and the Jacobian bucket array beyond the largest class that runs plan 0.
// Every size class up to the capacity must be tuned (a serving lane's are) and
// no pipeline captured yet; a prover with a forced plan keeps everything.
void trim_working_set(vkzg_prover *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (p->plan_forced >= 0 || p->plan_of.empty() || !p->graphs.empty()) return;
    for (uint32_t c = 1; c < p->cap; c <<= 1)
        if (!p->plan_of.count(c)) return;
    if (!p->plan_of.count(size_class(p->cap))) return;
    if (cudaSetDevice(p->device) != cudaSuccess || cudaStreamSynchronize(p->stream) != cudaSuccess) return;
    bool batch_affine = false;
    uint32_t plan0 = 0;
    for (const auto &kv : p->plan_of) {
        batch_affine |= kv.second == 1 || kv.second == 2 || kv.second == 4;
        if (kv.second == 0) plan0 = std::max(plan0, std::min(kv.first, p->cap));
    }
    ProofWork &w = p->pw;
    // plan 3 stands in for any plan whose buffers go (plan_for): keep them all
    // unless the digit table and its buffers are in place
    if (!p->comb || !w.flat_dig || !w.flat_pre) return;
    if (!batch_affine && w.ba_scratch) p->release(w.ba_scratch);
    p->plan0_cap = p->cap;
    if (plan0 < p->cap && w.buckets) {
        p->release(w.buckets);
        p->plan0_cap = 0;
        if (plan0 && p->alloc(w.buckets, (size_t)plan0 * kCells * kBuckets)) p->plan0_cap = plan0;
    }
    p->trimmed = true;
}

void set_comb_budget(vkzg_prover *p, uint64_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mutex);
    p->comb_budget = bytes;
}

void adopt_tuning(vkzg_prover *dst, const vkzg_prover *src) {
    if (!dst || !src) return;
    std::lock_guard<std::mutex> lock(dst->mutex);
    if (cudaSetDevice(dst->device) != cudaSuccess) return;
    bool want_comb = false, want_flat = false;
    dst->comb_budget = src->comb_budget;
    dst->comb_windows_chosen = src->comb_windows_chosen;
    for (const auto &kv : src->plan_of) {
        dst->plan_of[kv.first] = kv.second;
        want_comb |= kv.second == 3;
        want_flat |= kv.second == 4;
    }
    if (want_comb) ensure_comb(dst);
    if (want_flat) ensure_flat_b(dst);
}
} // namespace vkzg

uint64_t vkzg_b200_kernel_launches(void) { return launches_total(); }

int vkzg_b200_digit_table(const vkzg_prover *p, double *build_ms, uint64_t *bytes) {
    if (!p || !p->comb) return 0;
    if (build_ms) *build_ms = p->comb->build_ms;
    if (bytes) *bytes = p->comb->bytes;
    return p->comb->windows;
}

void vkzg_b200_prover_device_bytes(const vkzg_prover *p, uint64_t *working, uint64_t *tables, uint64_t *digit_table) {
    if (working) *working = p ? p->dev_bytes - p->tables_bytes : 0;
    if (tables) *tables = p ? p->tables_bytes : 0;
    if (digit_table) *digit_table = p && p->comb ? p->comb->bytes : 0;
}

int vkzg_b200_window_trials(const vkzg_prover *p, uint32_t size_class, int *windows, uint64_t *table_bytes,
                            double *build_ms, double *ms, int cap) {
    if (!p) return 0;
    auto it = p->window_trials.find(size_class);
    if (it == p->window_trials.end()) return 0;
    int i = 0;
    for (const auto &t : it->second) {
        if (i < cap) {
            if (windows) windows[i] = t.windows;
            if (table_bytes) table_bytes[i] = t.bytes;
            if (build_ms) build_ms[i] = t.build_ms;
            if (ms) ms[i] = t.ms;
        }
        i++;
    }
    return i;
}

int vkzg_b200_tuning_table(const vkzg_prover *p, uint32_t *size_class_out, int *plan_out, double *ms_out, int cap) {
    if (!p) return 0;
    int i = 0;
    for (const auto &kv : p->plan_of) {
        if (i < cap) {
            if (size_class_out) size_class_out[i] = kv.first;
            if (plan_out) plan_out[i] = kv.second;
            auto it = p->plan_ms.find(kv.first);
            if (ms_out)
                for (int q = 0; q < kPlans; q++) {
                    const double v = it != p->plan_ms.end() ? it->second[q] : -1.0;
                    ms_out[kPlans * i + q] = v >= 1e29 ? -1.0 : v;
                }
        }
        i++;
    }
    return i;
}

// --------------------------------------- recovered cells and their proofs

// recover_cells_and_kzg_proofs: the extension is systematic, so the first 64
// cells of the recovered wire-order array are the blob itself (element i of
// that half sits at domain point w_8192^brev13(i) = w_4096^brev12(i)); proofs
// are computed from them after a device-to-device copy.  Pinned by the
// recovery vectors' proofs (output[1], which tests/vectors.h:8-10 skips).
vkzg_result vkzg_b200_recover_cells_and_proofs_batch(vkzg_prover *p, uint8_t *cells_out, uint8_t *proofs_out,
                                                     const uint8_t *cells, const uint8_t *cell_present,
                                                     size_t num_blobs) {
    if (!p || !cells_out || !proofs_out || !cells || !cell_present) return VKZG_ERR_BADARGS;
    if (num_blobs == 0) return VKZG_OK;
    std::lock_guard<std::mutex> lock(p->mutex);
    if (cudaSetDevice(p->device) != cudaSuccess) return VKZG_ERR_GPU;
    const size_t ext_bytes = (size_t)kExtElems * 32;
    for (size_t done = 0; done < num_blobs;) {
        const uint32_t n = (uint32_t)std::min<size_t>(p->cap, num_blobs - done);
        const uint8_t *pr = cell_present + done * kCells;
        for (uint32_t b = 0; b < n; b++) {
            int miss = 0;
            for (int i = 0; i < kCells; i++) miss += pr[(size_t)b * kCells + i] == 0;
            if (miss > kCellElems) return VKZG_ERR_BADARGS;
        }
        cudaStream_t s = p->stream;
        CK(cudaMemcpyAsync(p->rw.cells, cells + done * ext_bytes, (size_t)n * ext_bytes, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(p->rw.present, pr, (size_t)n * kCells, cudaMemcpyHostToDevice, s));
        CK(launch_recover_timed(p->t, p->rw, (int)n, s, nullptr));
        CK(cudaMemcpy2DAsync(p->pw.blobs, kBlobBytes, p->rw.out, ext_bytes, kBlobBytes, n, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemsetAsync(p->pw.err, 0, n * sizeof(uint32_t), s));
        p->pw.plan = plan_for(p, n);
        CK(run_proofs(p, p->pw, n));
        CK(cudaMemcpyAsync(cells_out + done * ext_bytes, p->rw.out, (size_t)n * ext_bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(proofs_out + done * kCells * kProofBytes, p->pw.proofs, (size_t)n * kCells * kProofBytes,
                           cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        done += n;
    }
    return VKZG_OK;
}
