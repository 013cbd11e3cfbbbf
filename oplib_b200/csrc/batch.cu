// Batched solve of many uneven lattices (the calibration-sweep workload).
//
// Precedent: the reference's grouped GEMM runs many matrices of different sizes in one
// launch through a per-block task table (oplib/opcuda/sgemm4.cu:84-154), and its planner
// batches every interval that still needs squaring at level r into one call
// (oplib/opmodel/models/CModel Common.cs:508-545, CModel Device.cs:216-228).  Here every
// squaring level of all lattices is ONE persistent tcgen05 launch over a work list of
// (lattice, m-tile, n-tile) items.  Its epilogue writes the next level's 16-bit parts and
// applies the previous level's deferred FP64 row normalisation, so between levels only a
// small row-fix launch runs (plus a renormalisation of the lattices whose last level it
// was); chaining and pricing are batched the same way.  The plan (tables, tensor maps, work
// lists) is built once on the host and uploaded into the caller's workspace; execute()
// then issues 2-4 launches per level with no host synchronisation and no allocation, so a
// whole sweep can be captured in a CUDA graph and replayed.
//
// Tile shape and work order are chosen by opb_batch_autotune, which times the chain
// product for each candidate (tile width 64, 128, 256 or 256 on CTA pairs; items ordered
// longest-K first or by lattice) with CUDA events and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "lattice.h"

enum { OPB_FP32_PLAIN_B = 0, OPB_FP32_RENORM_B = 1, OPB_BF16X3_B = 2, OPB_FP16X3_B = 3 };
static inline bool tc_mode_b(int m) { return m == OPB_BF16X3_B || m == OPB_FP16X3_B; }
static constexpr float F16S = 32768.f;  // split scale of FP16 parts (|E|, P <= 1)

struct opb_lattice_desc;  // lattice.cu
extern "C" int opb_lattice_solve(const opb_lattice_desc *L, int mode, void *workspace, unsigned long long ws_bytes,
                                 double *quotes, double *V_all);
extern "C" unsigned long long opb_lattice_workspace_size(int d, int nK, int mode);
extern "C" int opb_lattice_bermudan(const opb_lattice_desc *L, int mode, int put, int exercise, double barrier,
                                    void *workspace, unsigned long long ws_bytes, double *quotes);

struct opb_batch_desc {
    int nlat;
    const int *d;            // host [nlat], multiples of 128
    const int *y0;           // host [nlat]
    const int *niter;        // host [nlat], >= 1
    const double *dt;        // host [nlat]
    const double *rate;      // host [nlat]
    int ell_width;
    const int *gen_cols;     // device [sum(d) * ell_width], columns within the lattice
    const double *gen_vals;  // device [sum(d) * ell_width]
    const double *x;         // device [sum(d)]
    int nmat;
    double period;
    int nK;
    const double *strikes;   // device [nlat * nK]
};

namespace {

// (bn, order): (128, LPT), (64, LPT), (128, lattice), (64, lattice), (256 mixed, LPT),
// (256 mixed, lattice), (256 pair mixed, LPT), (256 pair mixed, lattice).  "256 mixed":
// 128 x 256 tiles for the lattices whose size is a multiple of 256, 128 x 128 tiles for
// the rest (two launches per level); "256 pair mixed": 256 x 256 tiles on 2-CTA clusters
// for those lattices instead.
constexpr int NCFG = 8;
constexpr int CFG_BN[NCFG] = {128, 64, 128, 64, 256, 256, 256, 256};
constexpr bool CFG_PAIR[NCFG] = {false, false, false, false, false, false, true, true};

// mirror of opb_lattice_desc (lattice.cu), used for the FP32 per-lattice path
struct LatticeDescMirror {
    int d, y0, ell_width;
    const int *gen_cols;
    const double *gen_vals;
    const double *gen_dense;
    const double *x;
    double dt;
    int niter, nmat;
    double period, rate;
    int nK;
    const double *strikes;
};

struct ListRef {
    size_t off;  // element offset in the work blob
    int n;
};

}  // namespace

struct opb_batch_plan {
    int f16 = 0;
    int mode = 0, nlat = 0, nmat = 0, nK = 0, ldk = 64, maxn = 0, cfg = 0, grid = 0;
    long long total_rows = 0;
    int ell_width = 0;
    const int *cols = nullptr;
    const double *vals = nullptr, *x = nullptr, *strikes = nullptr;
    // lattices off the 128 grid (split modes): the caller's arrays, padded into these before
    // every execution (cols / vals / x then point to the padded copies)
    bool padded = false;
    const int *cols_src = nullptr;
    const double *vals_src = nullptr, *x_src = nullptr;
    int *cols_pad = nullptr;
    double *vals_pad = nullptr, *x_pad = nullptr;
    double period = 0.0;
    // device tables
    opb::BatchLattice *lats = nullptr;
    // the squaring and chain problems and maps come in two sets, [0] reading the parts in
    // the A buffers and [1] those in the other buffer (squarings: B; chains: the pair carved
    // from the FP32 chain buffer), each product writing its output's parts into the other
    opb::TcProblem *sq[2] = {nullptr, nullptr}, *chain[2] = {nullptr, nullptr}, *price = nullptr;
    opb::RenormProblem *rn_sq = nullptr;
    // 4 maps per lattice (Ahi, Alo, Bhi, Blo), the same for every tile width: squaring (B =
    // E's row-major parts, MN-major), chain (B = P1's row-major parts), pricing (K-major
    // payoff parts), per part set
    CUtensorMap *maps_sq[2] = {nullptr, nullptr}, *maps_ch[2] = {nullptr, nullptr}, *maps_price[2] = {nullptr, nullptr};
    __nv_bfloat16 *B_hi = nullptr, *B_lo = nullptr;  // the B part buffers of all lattices
    size_t B_bytes = 0;                                 // of each
    // backward induction: A = P1's parts, B = the option values' parts read d x ldk row-major
    CUtensorMap *maps_berm = nullptr;
    uint32_t *work = nullptr;
    float *E_base = nullptr;
    size_t E_bytes = 0;
    // work lists (offsets into `work`)
    std::vector<ListRef> gemm_level[NCFG];
    ListRef gemm_chain[NCFG];
    std::vector<ListRef> gemm_level_rest[NCFG];  // pair configurations: the 128 x 256 items
    ListRef gemm_chain_rest[NCFG];
    ListRef gemm_price;
    std::vector<ListRef> rn_level;     // per level: the lattices whose last level it is (P1)
    std::vector<char> level_inter;     // per level: some lattice squares on after it
    ListRef rn_init;
    // FP32 path
    std::vector<LatticeDescMirror> fp32_desc;
    std::vector<char *> fp32_ws;
    size_t fp32_ws_bytes = 0;
};

namespace {

struct Carve {
    char *base;
    size_t used;
    template <class T>
    T *take(size_t n) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + n * sizeof(T);
        return base ? reinterpret_cast<T *>(base + off) : nullptr;
    }
};

int check_batch(const opb_batch_desc *b, int mode) {
    if (!b) return OPB_E_NULL;
    if (b->nlat < 1 || b->nlat > 65535 || b->nmat < 1 || b->nK < 1 || b->nK > 64) return OPB_E_ARG;
    if (!b->d || !b->y0 || !b->niter || !b->dt || !b->rate) return OPB_E_NULL;
    if (!b->gen_cols || !b->gen_vals || !b->x || !b->strikes) return OPB_E_NULL;
    if (b->ell_width < 1 || !(b->period > 0.0)) return OPB_E_ARG;
    if (mode < 0 || mode > 3) return OPB_E_ARG;
    for (int i = 0; i < b->nlat; i++) {
        int d = b->d[i];
        if (d < 2 || d > 8064 || b->y0[i] < 0 || b->y0[i] >= d || b->niter[i] < 1 || !(b->dt[i] > 0.0))
            return OPB_E_ARG;
    }
    return OPB_OK;
}

// The split modes run every lattice on a multiple of 128 states: a lattice of another size
// is solved as one padded with absorbing states (zero generator rows and columns), whose
// rows of every product, renormalisation and price are the unpadded lattice's (no state of
// the lattice reaches a padding state).
std::vector<int> plan_sizes(const opb_batch_desc *b, int mode) {
    std::vector<int> d(b->d, b->d + b->nlat);
    if (tc_mode_b(mode))
        for (int &v : d) v = (v + 127) / 128 * 128;
    return d;
}

bool plan_padded(const opb_batch_desc *b, int mode) {
    if (!tc_mode_b(mode)) return false;
    for (int i = 0; i < b->nlat; i++)
        if (b->d[i] % 128) return true;
    return false;
}

// The layout works on the plan's (padded) sizes: a copy of the descriptor with them.
struct PlanDesc {
    std::vector<int> d;
    opb_batch_desc desc;
    PlanDesc(const opb_batch_desc *b, int mode) : d(plan_sizes(b, mode)), desc(*b) { desc.d = d.data(); }
};

// Layout of all device buffers and tables; with base == nullptr it only measures.
// K-blocks of 64 that a squaring tile (rows [m0, m0 + tm), columns [n0, n0 + tn)) issues at
// `level` when the generator's half-bandwidth is h0 (0: unknown, dense): the host mirror of
// the kernel's band_kblocks with its 128-wide accumulation chunks, used to order the work.
int host_band_kblocks(int h0, int level, int m0, int tm, int n0, int tn, int K) {
    const int all = K / 64;
    if (h0 <= 0) return all;
    const long long h = level >= 40 ? (1LL << 40) : (long long)h0 << level;
    if (h >= K) return all;
    const long long lo = (long long)std::max(m0, n0) - h, hi = (long long)std::min(m0 + tm, n0 + tn) - 1 + h;
    if (lo > hi || hi < 0 || lo >= K) return 0;
    const int c_lo = (int)(std::max(lo, 0LL) / 128), c_hi = (int)(std::min(hi, (long long)K - 1) / 128) + 1;
    return std::min(2 * c_hi, all) - 2 * c_lo;
}

// bands: the generators' half-bandwidths (nullptr when only measuring): the squaring levels'
// work lists of the longest-first configurations are then ordered by the K-blocks each item
// issues at that level, longest first.
size_t layout(const opb_batch_desc *b, int mode, opb_batch_plan *P, char *base, std::vector<uint32_t> *work_out,
              const std::vector<int> *bands = nullptr, bool padded = false) {
    Carve c{base, 0};
    const int n = b->nlat;
    std::vector<long long> off(n + 1, 0);
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + b->d[i];
    if (!tc_mode_b(mode)) {
        size_t per_max = 0;
        std::vector<size_t> sz(n);
        for (int i = 0; i < n; i++) {
            sz[i] = opb_lattice_workspace_size(b->d[i], b->nK, mode);
            per_max = std::max(per_max, sz[i]);
        }
        // lattices are solved one after another on one stream, so one workspace suffices
        char *ws = c.take<char>(per_max);
        if (P) {
            P->fp32_ws.assign(1, ws);
            P->fp32_ws_bytes = per_max;
        }
        return c.used + 256;
    }
    const int ldk = 64;
    auto lats = c.take<opb::BatchLattice>(n);
    auto sq = c.take<opb::TcProblem>(2 * (size_t)n);
    auto ch = c.take<opb::TcProblem>(2 * (size_t)n);
    auto pr = c.take<opb::TcProblem>(n);
    auto rs = c.take<opb::RenormProblem>(n);
    auto msq = c.take<CUtensorMap>(8 * (size_t)n);
    auto mch = c.take<CUtensorMap>(8 * (size_t)n);
    auto mp = c.take<CUtensorMap>(8 * (size_t)n);
    size_t Etot = 0;
    for (int i = 0; i < n; i++) Etot += (size_t)b->d[i] * b->d[i];
    float *E = c.take<float>(Etot);
    float *Pa = c.take<float>(Etot);
    __nv_bfloat16 *Ah = c.take<__nv_bfloat16>(Etot), *Al = c.take<__nv_bfloat16>(Etot);
    __nv_bfloat16 *Bh = c.take<__nv_bfloat16>(Etot), *Bl = c.take<__nv_bfloat16>(Etot);
    float *V = c.take<float>((size_t)off[n] * ldk);
    __nv_bfloat16 *Gh = c.take<__nv_bfloat16>((size_t)off[n] * ldk), *Gl = c.take<__nv_bfloat16>((size_t)off[n] * ldk);
    size_t parts = 0;
    for (int i = 0; i < n; i++) parts += (size_t)(b->d[i] / 64) * b->d[i];
    double *part = c.take<double>(parts);
    (void)c.take<float>(n);          // per-lattice FP16 payoff scales
    (void)c.take<double2>(off[n]);   // per-row fixes of the deferred E-form renormalisation
    auto mbm = c.take<CUtensorMap>(4 * (size_t)n);  // backward-induction maps
    (void)c.take<double>((size_t)off[n] * ldk);     // FP64 option values of the backward induction

    // ---- work lists (host), appended into one blob
    std::vector<uint32_t> W;
    std::vector<int> lpt(n), nat(n);
    std::iota(nat.begin(), nat.end(), 0);
    lpt = nat;
    std::stable_sort(lpt.begin(), lpt.end(), [&](int a, int bb) { return b->d[a] > b->d[bb]; });
    int maxn = 0;
    for (int i = 0; i < n; i++) maxn = std::max(maxn, b->niter[i]);
    // sel: 0 every lattice, 1 only sizes that are multiples of 256, 2 only the others.  A
    // size that is not a multiple of bn gets a last column tile that overhangs the matrix:
    // its B columns beyond d load as zeros and its output groups beyond d are not stored.
    auto gemm_list = [&](const std::vector<int> &order, int bn, int level, bool chain_or_all, int sel = 0,
                         int tile_m = 128, bool by_work = false) {
        ListRef r{W.size(), 0};
        for (int i : order) {
            if (!chain_or_all && b->niter[i] <= level) continue;
            if ((sel == 1 && b->d[i] % 256) || (sel == 2 && b->d[i] % 256 == 0)) continue;
            const int mt = b->d[i] / tile_m, nt = (b->d[i] + bn - 1) / bn;
            for (int a = 0; a < mt; a++)
                for (int bb = 0; bb < nt; bb++) W.push_back(((uint32_t)i << 16) | ((uint32_t)a << 8) | (uint32_t)bb);
        }
        r.n = (int)(W.size() - r.off);
        if (by_work && bands && !chain_or_all) {
            auto kb = [&](uint32_t w) {
                const int i = (int)(w >> 16);
                return host_band_kblocks((*bands)[i], level, (int)((w >> 8) & 255u) * tile_m, tile_m,
                                         (int)(w & 255u) * bn, bn, b->d[i]);
            };
            std::stable_sort(W.begin() + r.off, W.end(), [&](uint32_t x, uint32_t y) { return kb(x) > kb(y); });
        }
        return r;
    };
    std::vector<ListRef> gl[NCFG], glr[NCFG];
    ListRef gch[NCFG], gchr[NCFG];
    for (int cfg = 0; cfg < NCFG; cfg++) {
        const bool longest = cfg < 2 || cfg == 4 || cfg == 6;
        const auto &order = longest ? lpt : nat;
        if (CFG_PAIR[cfg]) {
            // 256 x 256 pair items for the multiples of 256, then 128 x 256 items (column
            // overhang) for the other sizes
            for (int lv = 0; lv < maxn; lv++) {
                gl[cfg].push_back(gemm_list(order, 256, lv, false, 1, 256, longest));
                glr[cfg].push_back(gemm_list(order, 256, lv, false, 2, 128, longest));
            }
            gch[cfg] = gemm_list(order, 256, 0, true, 1, 256);
            gchr[cfg] = gemm_list(order, 256, 0, true, 2, 128);
        } else {
            for (int lv = 0; lv < maxn; lv++) {
                gl[cfg].push_back(gemm_list(order, CFG_BN[cfg], lv, false, 0, 128, longest));
                glr[cfg].push_back(ListRef{W.size(), 0});
            }
            gch[cfg] = gemm_list(order, CFG_BN[cfg], 0, true);
            gchr[cfg] = ListRef{W.size(), 0};
        }
    }
    ListRef gpr{W.size(), 0};
    for (int i : lpt)
        for (int a = 0; a < b->d[i] / 128; a++) W.push_back(((uint32_t)i << 16) | ((uint32_t)a << 8));
    gpr.n = (int)(W.size() - gpr.off);
    auto rn_list = [&](int level, int kind) {  // kind: 0 init split, 1 the lattices ending at `level`
        ListRef r{W.size(), 0};
        for (int i : lpt) {
            int mode_i = 0;
            if (kind == 1) {
                if (b->niter[i] != level + 1) continue;
                mode_i = 1;
            }
            const int t = b->d[i] / 64, nch = opb::renorm_chunks(b->d[i]);
            for (int a = 0; a < t; a++)
                for (int c = 0; c < nch; c++)
                    W.push_back(((uint32_t)i << 16) | ((uint32_t)mode_i << 14) | ((uint32_t)a << 7) | (uint32_t)c);
        }
        r.n = (int)(W.size() - r.off);
        return r;
    };
    ListRef rinit = rn_list(0, 0);
    std::vector<ListRef> rl;
    std::vector<char> inter(maxn, 0);
    for (int lv = 0; lv < maxn; lv++) {
        rl.push_back(rn_list(lv, 1));
        for (int i = 0; i < n; i++) inter[lv] |= b->niter[i] > lv + 1 ? 1 : 0;
    }
    uint32_t *work = c.take<uint32_t>(W.size());
    // padded copies of the generator and spot values (lattices off the 128 grid)
    int *cols_pad = nullptr;
    double *vals_pad = nullptr, *x_pad = nullptr;
    if (padded) {
        cols_pad = c.take<int>((size_t)off[n] * b->ell_width);
        vals_pad = c.take<double>((size_t)off[n] * b->ell_width);
        x_pad = c.take<double>((size_t)off[n]);
    }
    size_t total = c.used + 256;
    if (!P) return total;
    P->padded = padded;
    P->cols_pad = cols_pad; P->vals_pad = vals_pad; P->x_pad = x_pad;

    // ---- fill the plan and host copies of the tables
    P->nlat = n; P->nmat = b->nmat; P->nK = b->nK; P->ldk = ldk; P->maxn = maxn;
    P->total_rows = off[n]; P->ell_width = b->ell_width; P->cols = b->gen_cols; P->vals = b->gen_vals;
    P->x = b->x; P->strikes = b->strikes; P->period = b->period;
    P->lats = lats; P->sq[0] = sq; P->sq[1] = sq + n; P->chain[0] = ch; P->chain[1] = ch + n; P->price = pr;
    P->rn_sq = rs;
    for (int k = 0; k < 2; k++) {
        P->maps_sq[k] = msq + 4 * (size_t)n * k;
        P->maps_ch[k] = mch + 4 * (size_t)n * k;
        P->maps_price[k] = mp + 4 * (size_t)n * k;
    }
    P->maps_berm = mbm; P->work = work;
    P->B_hi = Bh; P->B_lo = Bl; P->B_bytes = sizeof(__nv_bfloat16) * Etot;
    P->E_base = E; P->E_bytes = Etot * sizeof(float);
    for (int cfg = 0; cfg < NCFG; cfg++) {
        P->gemm_level[cfg] = gl[cfg];
        P->gemm_chain[cfg] = gch[cfg];
        P->gemm_level_rest[cfg] = glr[cfg];
        P->gemm_chain_rest[cfg] = gchr[cfg];
    }
    P->gemm_price = gpr; P->rn_level = rl; P->level_inter = inter; P->rn_init = rinit;
    if (work_out) *work_out = W;
    return total;
}

}  // namespace

using opb::set_status;

OPB_API unsigned long long opb_batch_workspace_size(const opb_batch_desc *b, int mode) {
    if (check_batch(b, mode) != OPB_OK) return 0;
    PlanDesc pd(b, mode);
    return (unsigned long long)layout(&pd.desc, mode, nullptr, nullptr, nullptr, nullptr, plan_padded(b, mode));
}

// Builds the plan: tables, tensor maps and work lists are written into `workspace`
// (blocking copies; call once, before any capture).  *out receives a host handle.
OPB_API int opb_batch_plan_create(const opb_batch_desc *b, int mode, void *workspace, unsigned long long ws_bytes,
                                  opb_batch_plan **out) {
    int c = check_batch(b, mode);
    if (c != OPB_OK) return set_status(c);
    OPB_REQUIRE(workspace && out, OPB_E_NULL);
    const bool padded = plan_padded(b, mode);
    PlanDesc pd(b, mode);
    size_t need = layout(&pd.desc, mode, nullptr, nullptr, nullptr, nullptr, padded);
    OPB_REQUIRE(ws_bytes >= need, OPB_E_ARG);
    char *base = reinterpret_cast<char *>(workspace);
    base += (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    opb_batch_plan *P = new opb_batch_plan();
    P->mode = mode;
    const int n = b->nlat;
    // the generators' half-bandwidths, from their column pattern (read once: the plan stays
    // valid while the generators' values change, not their columns)
    std::vector<int> bands(n, 0);
    if (tc_mode_b(mode)) {
        long long rows = 0;
        for (int i = 0; i < n; i++) rows += b->d[i];
        std::vector<int> cols((size_t)rows * b->ell_width);
        cudaError_t e = cudaMemcpyAsync(cols.data(), b->gen_cols, sizeof(int) * cols.size(), cudaMemcpyDeviceToHost,
                                        opb::stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(opb::stream());
        if (e != cudaSuccess) {
            delete P;
            return opb::set_cuda(e);
        }
        long long ro = 0;
        for (int i = 0; i < n; i++) {
            int h = 0;
            for (int y = 0; y < b->d[i]; y++)
                for (int k = 0; k < b->ell_width; k++) {
                    const int z = cols[(size_t)(ro + y) * b->ell_width + k];
                    if (z >= 0 && z < b->d[i]) h = std::max(h, std::abs(z - y));
                }
            bands[i] = h;
            ro += b->d[i];
        }
    }
    // from here on the plan's (padded) sizes; cb keeps the caller's
    const opb_batch_desc *cb = b;
    b = &pd.desc;
    std::vector<uint32_t> W;
    layout(b, mode, P, base, &W, &bands, padded);
    if (padded) {
        P->cols_src = cb->gen_cols; P->vals_src = cb->gen_vals; P->x_src = cb->x;
        P->cols = P->cols_pad; P->vals = P->vals_pad; P->x = P->x_pad;
    }
    if (!tc_mode_b(mode)) {
        P->nlat = n; P->nmat = b->nmat; P->nK = b->nK;
        long long roff = 0;
        for (int i = 0; i < n; i++) {
            LatticeDescMirror L{};
            L.d = b->d[i]; L.y0 = b->y0[i]; L.ell_width = b->ell_width;
            L.gen_cols = b->gen_cols + roff * b->ell_width; L.gen_vals = b->gen_vals + roff * b->ell_width;
            L.x = b->x + roff; L.dt = b->dt[i]; L.niter = b->niter[i]; L.nmat = b->nmat; L.period = b->period;
            L.rate = b->rate[i]; L.nK = b->nK; L.strikes = b->strikes + (size_t)i * b->nK;
            P->fp32_desc.push_back(L);
            roff += b->d[i];
        }
        *out = P;
        return set_status(OPB_OK);
    }
    // host images of the device tables
    std::vector<opb::BatchLattice> lats(n);
    std::vector<opb::TcProblem> sq(2 * (size_t)n), ch(2 * (size_t)n), pr(n);
    std::vector<opb::RenormProblem> rs(n);
    std::vector<CUtensorMap> msq(8 * (size_t)n), mch(8 * (size_t)n), mp(8 * (size_t)n), mbm(4 * (size_t)n);
    // recompute buffer pointers exactly as layout() carved them
    Carve cv{base, 0};
    cv.take<opb::BatchLattice>(n); cv.take<opb::TcProblem>(2 * (size_t)n); cv.take<opb::TcProblem>(2 * (size_t)n);
    cv.take<opb::TcProblem>(n); cv.take<opb::RenormProblem>(n);
    cv.take<CUtensorMap>(8 * (size_t)n); cv.take<CUtensorMap>(8 * (size_t)n); cv.take<CUtensorMap>(8 * (size_t)n);
    size_t Etot = 0;
    for (int i = 0; i < n; i++) Etot += (size_t)b->d[i] * b->d[i];
    float *E = cv.take<float>(Etot), *Pa = cv.take<float>(Etot);
    __nv_bfloat16 *Ah = cv.take<__nv_bfloat16>(Etot), *Al = cv.take<__nv_bfloat16>(Etot);
    __nv_bfloat16 *Bh = cv.take<__nv_bfloat16>(Etot), *Bl = cv.take<__nv_bfloat16>(Etot);
    float *V = cv.take<float>((size_t)P->total_rows * P->ldk);
    __nv_bfloat16 *Gh = cv.take<__nv_bfloat16>((size_t)P->total_rows * P->ldk);
    __nv_bfloat16 *Gl = cv.take<__nv_bfloat16>((size_t)P->total_rows * P->ldk);
    size_t parts = 0;
    for (int i = 0; i < n; i++) parts += (size_t)(b->d[i] / 64) * b->d[i];
    double *part = cv.take<double>(parts);
    float *gsc = cv.take<float>(n);
    double2 *fix = cv.take<double2>((size_t)P->total_rows);
    (void)cv.take<CUtensorMap>(4 * (size_t)n);
    double *vd = cv.take<double>((size_t)P->total_rows * P->ldk);
    const int f16 = mode == OPB_FP16X3_B ? 1 : 0;
    P->f16 = f16;
    const float un2 = f16 ? 1.f / (F16S * F16S) : 1.f, un1 = f16 ? 1.f / F16S : 1.f;
    size_t eo = 0, po = 0;
    long long ro = 0, so = 0;
    int rc_status = OPB_OK;
    for (int i = 0; i < n && rc_status == OPB_OK; i++) {
        const int d = b->d[i];
        const size_t dd = (size_t)d * d;
        opb::BatchLattice &L = lats[i];
        L.d = d; L.y0 = b->y0[i]; L.row_off = ro; L.dt = b->dt[i]; L.rate = b->rate[i]; L.period = b->period;
        L.d_src = cb->d[i]; L.src_off = so;
        so += cb->d[i];
        L.E = E + eo; L.Pa = Pa + eo; L.V = V + (size_t)ro * P->ldk;
        L.GThi = Gh + (size_t)ro * P->ldk; L.GTlo = Gl + (size_t)ro * P->ldk;
        L.gscale = gsc + i;
        L.Vd = vd + (size_t)ro * P->ldk;
        double *pi = part + po;
        L.niter = b->niter[i]; L.partial = pi; L.fix = fix + ro;
        // part sets: squarings between A and B, chains between A and a pair carved from the
        // FP32 chain buffer (2 d^2 BF16 values in its d^2 floats)
        __nv_bfloat16 *sh[2] = {Ah + eo, Bh + eo}, *sl[2] = {Al + eo, Bl + eo};
        __nv_bfloat16 *c2 = reinterpret_cast<__nv_bfloat16 *>(Pa + eo);
        __nv_bfloat16 *chh[2] = {Ah + eo, c2}, *chl[2] = {Al + eo, c2 + dd};
        for (int k = 0; k < 2 && rc_status == OPB_OK; k++) {
            // squaring: E' = 2E + E.E in place of E (as the previous level's GEMM left it, its
            // normalisation deferred into this epilogue through the row fixes), the output's
            // parts into the other set
            sq[k * n + i] = opb::TcProblem{d, d, d, bands[i], L.E, L.E, pi, d, un2, 2.f, fix + ro, sh[k ^ 1],
                                           sl[k ^ 1]};
            // chain: parts only, P_{m-1}'s row fix applied in the epilogue
            ch[k * n + i] = opb::TcProblem{d, d, d, 0, nullptr, nullptr, pi, d, un2, 0.f, fix + ro, chh[k ^ 1],
                                           chl[k ^ 1]};
            rc_status = opb::tc_make_maps(&msq[4 * ((size_t)k * n + i)], sh[k], sl[k], d, d, sh[k], sl[k], d, d, d,
                                          64, f16, 1);
            if (rc_status == OPB_OK)
                rc_status = opb::tc_make_maps(&mch[4 * ((size_t)k * n + i)], chh[k], chl[k], d, d, Bh + eo, Bl + eo, d,
                                              d, d, 64, f16, 1);
            if (rc_status == OPB_OK)
                rc_status = opb::tc_make_maps(&mp[4 * ((size_t)k * n + i)], chh[k], chl[k], d, d, L.GThi, L.GTlo,
                                              P->ldk, d, d, 64, f16);
        }
        pr[i] = opb::TcProblem{d, P->ldk, d, 0, L.V, nullptr, nullptr, P->ldk, un1, 0.f, nullptr};
        rs[i] = opb::RenormProblem{d, 0, L.E, pi, Ah + eo, Al + eo, Bh + eo, Bl + eo, fix + ro};
        if (rc_status == OPB_OK)  // the same buffers, the value parts read d x ldk row-major
            rc_status = opb::tc_make_maps(&mbm[4 * (size_t)i], Ah + eo, Al + eo, d, d, L.GThi, L.GTlo, P->ldk,
                                          P->ldk, d, 64, f16, 1);
        eo += dd;
        po += (size_t)(d / 64) * d;
        ro += d;
    }
    if (rc_status != OPB_OK) {
        delete P;
        return set_status(rc_status);
    }
    // uploads on the library stream (ordered after any earlier work on the workspace), then
    // one synchronisation before the host staging vectors go out of scope
    cudaStream_t ls = opb::stream();
    auto up = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ls);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up(P->lats, lats.data(), sizeof(opb::BatchLattice) * n);
    if (e == cudaSuccess) e = up(P->sq[0], sq.data(), sizeof(opb::TcProblem) * 2 * (size_t)n);
    if (e == cudaSuccess) e = up(P->chain[0], ch.data(), sizeof(opb::TcProblem) * 2 * (size_t)n);
    if (e == cudaSuccess) e = up(P->price, pr.data(), sizeof(opb::TcProblem) * n);
    if (e == cudaSuccess) e = up(P->rn_sq, rs.data(), sizeof(opb::RenormProblem) * n);
    if (e == cudaSuccess) e = up(P->maps_sq[0], msq.data(), sizeof(CUtensorMap) * 8 * (size_t)n);
    if (e == cudaSuccess) e = up(P->maps_ch[0], mch.data(), sizeof(CUtensorMap) * 8 * (size_t)n);
    if (e == cudaSuccess) e = up(P->maps_price[0], mp.data(), sizeof(CUtensorMap) * 8 * (size_t)n);
    if (e == cudaSuccess) e = up(P->maps_berm, mbm.data(), sizeof(CUtensorMap) * 4 * (size_t)n);
    if (e == cudaSuccess) e = up(P->work, W.data(), sizeof(uint32_t) * W.size());
    const cudaError_t es = cudaStreamSynchronize(ls);
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) {
        delete P;
        return opb::set_cuda(e);
    }
    P->cfg = 0;
    P->grid = 0;
    *out = P;
    return set_status(OPB_OK);
}

OPB_API int opb_batch_num_configs(void) { return NCFG; }

OPB_API int opb_batch_plan_destroy(opb_batch_plan *P) {
    delete P;
    return set_status(OPB_OK);
}

// Selects the launch configuration: cfg 0..7 = (BN 128, longest-K first), (64, longest
// first), (128, lattice order), (64, lattice order), (128 x 256 tiles for every size,
// longest first), (the same, lattice order), (256 x 256 pair items for the multiples of
// 256 and 128 x 256 tiles for the rest, longest first), (the same, lattice order); grid 0
// = one CTA per SM (the pair launches size their own grid).
OPB_API int opb_batch_set_config(opb_batch_plan *P, int cfg, int grid) {
    OPB_REQUIRE(P, OPB_E_NULL);
    OPB_REQUIRE(cfg >= 0 && cfg < NCFG && grid >= 0, OPB_E_ARG);
    P->cfg = cfg;
    P->grid = grid;
    return set_status(OPB_OK);
}

namespace {

// One squaring level (or the chain product) under configuration cfg: one launch, or two
// for the pair configurations (256 x 256 pair items, then 128 x 256 ones).  maps: the
// squaring or the chain table (MN-major B); fixmode: how the problems' row fixes apply.
int cfg_gemm(opb_batch_plan *P, int cfg, const CUtensorMap *maps, const opb::TcProblem *probs, const ListRef &l,
             const ListRef &rest, cudaStream_t s, int level, int lolo, int skip, int fixmode, int fuse) {
    const int bn = CFG_BN[cfg];
    const float ss = P->f16 ? F16S : 0.f;
    int r = CFG_PAIR[cfg] ? opb::launch_tc_gemm_batched_pair(maps, probs, P->work + l.off, l.n, s, P->f16, 1, level,
                                                             lolo, skip, fixmode, ss, fuse)
                          : opb::launch_tc_gemm_batched(bn, maps, probs, P->work + l.off, l.n, P->grid, s, P->f16, 1,
                                                        level, lolo, skip, fixmode, ss, fuse);
    if (r == 0 && rest.n > 0)
        r = opb::launch_tc_gemm_batched(256, maps, probs, P->work + rest.off, rest.n, P->grid, s, P->f16, 1, level,
                                        lolo, skip, fixmode, ss, fuse);
    return r;
}

// Squaring level `level` of every lattice still squaring; each lattice's operands are
// banded by its generator (TcProblem::band), and BF16 parts add the lo.lo product on the
// first OPB_LOLO_LEVELS levels, as in the single-lattice solve.  The level reads the part
// set level % 2 and writes the other; from level 1 on, the previous level's normalisation
// is deferred into this epilogue.
int level_gemm(opb_batch_plan *P, int cfg, int level, cudaStream_t s) {
    const int lolo = (!P->f16 && level < opb::g_lolo_levels) ? 1 : 0;
    const int k = level & 1;
    return cfg_gemm(P, cfg, P->maps_sq[k], P->sq[k], P->gemm_level[cfg][level], P->gemm_level_rest[cfg][level], s,
                    level, lolo, opb::g_band_skip, level > 0 ? opb::OPB_FIX_SQUARE : opb::OPB_FIX_NONE, 1);
}

// The chain product of every lattice (dense, all lattices active): what the autotuner times.
// set: the part set holding P_{m-1}; scaled: apply P_{m-1}'s row fixes (every chain but the
// first, whose A is the normalised P1).
int chain_gemm(opb_batch_plan *P, int cfg, cudaStream_t s, int set = 0, bool scaled = false) {
    return cfg_gemm(P, cfg, P->maps_ch[set], P->chain[set], P->gemm_chain[cfg], P->gemm_chain_rest[cfg], s, 0, 0, 0,
                    scaled ? opb::OPB_FIX_ROWSCALE : opb::OPB_FIX_NONE, 2);
}

// E0 build and every squaring level: P1 of every lattice as row-major parts in its A and B
// buffers.  Per level one GEMM, then the row fixes of the lattices that square on and the
// renormalisation (to P1) of those whose last level it was.
int batch_square(opb_batch_plan *P, cudaStream_t s) {
    const int cfg = P->cfg, bn = CFG_BN[cfg], pdiv = bn < 128 ? bn : 128;
    const float ss = P->f16 ? F16S : 0.f;
    int r = 0;
    // lattices off the 128 grid: the caller's generators and spot values into the padded rows
    // (every execution: a calibration rewrites the generators' values between runs)
    if (P->padded)
        r = opb::launch_pad_batched(P->lats, P->nlat, P->total_rows, P->ell_width, P->cols_src, P->vals_src,
                                    P->x_src, P->cols_pad, P->vals_pad, P->x_pad, s);
    if (r == 0) r = (int)cudaMemsetAsync(P->E_base, 0, P->E_bytes, s);
    // the B part set starts zeroed: a level skips the output tiles outside its operands'
    // band, which must read as zeros when the next level issues their K-blocks
    if (r == 0) r = (int)cudaMemsetAsync(P->B_hi, 0, P->B_bytes, s);
    if (r == 0) r = (int)cudaMemsetAsync(P->B_lo, 0, P->B_bytes, s);
    if (r == 0) r = opb::launch_ek_batched(P->lats, P->nlat, P->total_rows, P->ell_width, P->cols, P->vals, s);
    if (r == 0) r = opb::launch_renorm_batched(P->rn_sq, P->work + P->rn_init.off, P->rn_init.n, 0, s, ss);
    for (int lv = 0; lv < P->maxn && r == 0; lv++) {
        r = level_gemm(P, cfg, lv, s);
        if (r == 0 && P->level_inter[lv])
            r = opb::launch_rowfix_batched(P->lats, P->nlat, P->total_rows, pdiv, lv, 1, s);
        if (r == 0 && P->rn_level[lv].n > 0)
            r = opb::launch_renorm_batched(P->rn_sq, P->work + P->rn_level[lv].off, P->rn_level[lv].n, pdiv, s, ss);
    }
    return r;
}

}  // namespace

// Executes the plan on the library stream: E0 build, every squaring level (one GEMM +
// one renormalisation launch each), chaining and pricing.  quotes: device
// [nlat][nmat][nK] FP64.  No host synchronisation, no allocation (graph-capturable).
OPB_API int opb_batch_execute(opb_batch_plan *P, double *quotes) {
    OPB_NVTX("opb_batch_execute");
    OPB_REQUIRE(P && quotes, OPB_E_NULL);
    cudaStream_t s = opb::stream();
    int r = 0;
#define BT(expr)                                  \
    do {                                          \
        r = (expr);                               \
        if (r != 0) return set_status(r);         \
    } while (0)
    if (!tc_mode_b(P->mode)) {
        for (int i = 0; i < P->nlat; i++)
            BT(opb_lattice_solve(reinterpret_cast<const opb_lattice_desc *>(&P->fp32_desc[i]), P->mode, P->fp32_ws[0],
                                 P->fp32_ws_bytes, quotes + (size_t)i * P->nmat * P->nK, nullptr));
        return set_status(OPB_OK);
    }
    const int cfg = P->cfg, bn = CFG_BN[cfg], pdiv = bn < 128 ? bn : 128;
    BT(batch_square(P, s));
    BT(opb::launch_payoff_batched(P->lats, P->nlat, P->total_rows, P->nK, P->ldk, P->x, P->strikes, s, P->f16));
    // chains: P_m = P_{m-1} . P1 writes only its parts (into the other part set) and its row
    // sums; its row fixes scale the next chain's epilogue and this maturity's quotes
    int set = 0;
    for (int m = 1; m <= P->nmat; m++) {
        if (m > 1) {
            BT(chain_gemm(P, cfg, s, set, m > 2));
            BT(opb::launch_rowfix_batched(P->lats, P->nlat, P->total_rows, pdiv, -1, 0, s));
            set ^= 1;
        }
        BT(opb::launch_tc_gemm_batched(64, P->maps_price[set], P->price, P->work + P->gemm_price.off,
                                       P->gemm_price.n, P->grid, s, P->f16, 0));
        BT(opb::launch_quotes_batched(P->lats, P->nlat, P->nK, P->ldk, m, P->nmat, quotes, s, P->f16, m > 1));
    }
#undef BT
    return set_status(OPB_OK);
}

// Bermudan or barrier calls/puts on every lattice of the plan by backward induction on its
// period kernel (as opb_lattice_bermudan): maturity nmat * period, exercisable at every
// m * period (exercise = 1), knocked out at or below barrier on those dates (barrier >
// 0).  The squarings run as in opb_batch_execute; then per date one batched tensor-core
// product P1_i . V_i over all lattices and one FP64 step.  quotes: device [nlat][nK] FP64,
// the values at each lattice's y0.  No host synchronisation, no allocation.
OPB_API int opb_batch_execute_bermudan(opb_batch_plan *P, int put, int exercise, double barrier, double *quotes) {
    OPB_NVTX("opb_batch_execute_bermudan");
    OPB_REQUIRE(P && quotes, OPB_E_NULL);
    OPB_REQUIRE(put >= 0 && put <= 1 && exercise >= 0 && exercise <= 1 && barrier >= 0.0, OPB_E_ARG);
    cudaStream_t s = opb::stream();
    int r = 0;
#define BT(expr)                                  \
    do {                                          \
        r = (expr);                               \
        if (r != 0) return set_status(r);         \
    } while (0)
    if (!tc_mode_b(P->mode)) {
        for (int i = 0; i < P->nlat; i++)
            BT(opb_lattice_bermudan(reinterpret_cast<const opb_lattice_desc *>(&P->fp32_desc[i]), P->mode, put,
                                    exercise, barrier, P->fp32_ws[0], P->fp32_ws_bytes, quotes + (size_t)i * P->nK));
        return set_status(OPB_OK);
    }
    BT(batch_square(P, s));
    BT(opb::launch_berm_batched_init(P->lats, P->nlat, P->total_rows, P->nK, P->ldk, P->x, P->strikes, put, barrier,
                                     P->f16, s));
    for (int m = P->nmat - 1; m >= 0; m--) {
        BT(opb::launch_tc_gemm_batched(64, P->maps_berm, P->price, P->work + P->gemm_price.off, P->gemm_price.n,
                                       P->grid, s, P->f16, 1));
        BT(opb::launch_berm_batched_step(P->lats, P->nlat, P->total_rows, P->nK, P->ldk, P->x, P->strikes, put,
                                         barrier, exercise, m == 0, P->f16, quotes, s));
    }
#undef BT
    return set_status(OPB_OK);
}

// Times the chain product (dense, all lattices active: the shape of every squaring level
// once the operands have filled in) for every configuration with CUDA events and keeps the
// fastest; ms[cfg] (optional, opb_batch_num_configs() entries) receives the times.
// Blocking; leaves the plan's buffers in an arbitrary state (run execute afterwards).
OPB_API int opb_batch_autotune(opb_batch_plan *P, int reps, float *ms_out, int *best_cfg) {
    OPB_REQUIRE(P, OPB_E_NULL);
    if (!tc_mode_b(P->mode)) {
        if (best_cfg) *best_cfg = 0;
        return set_status(OPB_OK);
    }
    if (reps < 1) reps = 1;
    cudaStream_t s = opb::stream();
    cudaEvent_t e0, e1;
    OPB_TRY(cudaEventCreate(&e0));
    OPB_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    int bc = 0;
    for (int cfg = 0; cfg < NCFG; cfg++) {
        int r = chain_gemm(P, cfg, s);  // warm-up (also sets the smem attribute)
        if (r) return set_status(r);
        OPB_TRY(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; i++) {
            r = chain_gemm(P, cfg, s);
            if (r) return set_status(r);
        }
        OPB_TRY(cudaEventRecord(e1, s));
        OPB_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        OPB_TRY(cudaEventElapsedTime(&ms, e0, e1));
        ms /= reps;
        if (ms_out) ms_out[cfg] = ms;
        if (ms < best) { best = ms; bc = cfg; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P->cfg = bc;
    if (best_cfg) *best_cfg = bc;
    return set_status(OPB_OK);
}

// Launch counts of one execute() (library kernels and memsets), for accounting.
OPB_API int opb_batch_launches(const opb_batch_plan *P) {
    if (!P) return 0;
    if (!tc_mode_b(P->mode)) return -1;
    int extra = 0;  // the pair configurations' second GEMM launch per level / chain
    for (int lv = 0; lv < P->maxn; lv++) extra += P->gemm_level_rest[P->cfg][lv].n > 0 ? 1 : 0;
    if (P->gemm_chain_rest[P->cfg].n > 0) extra += P->nmat - 1;
    int per_level = 0;  // GEMM, row fixes (some lattice squares on), renormalisation (some ends)
    for (int lv = 0; lv < P->maxn; lv++)
        per_level += 1 + (P->level_inter[lv] ? 1 : 0) + (P->rn_level[lv].n > 0 ? 1 : 0);
    return 5 + (P->padded ? 1 : 0) + per_level + 1 + (P->f16 ? 1 : 0) + 2 * P->nmat + 2 * (P->nmat - 1) + extra;
}
