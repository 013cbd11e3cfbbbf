// Lattice solve: U0 = I + dt*L (FP64 build) -> niter squarings -> chaining to nmat
// maturities -> backward induction of call payoffs -> FP64 discounting -> quotes.
//
// This is the device half of the reference's CModel.exe_mc_plan on the device branch
// (oplib/opmodel/models/CModel Common.cs:651-669 -> device_mc_sfex, sminit, smk, smcopy;
// CModel Device.cs:186-295), restated for one interval length (period) and a maturity
// ladder T_m = m * period, m = 1..nmat, plus the payoff induction V_m = P(T_m) . G that
// the reference exposes as sgemv kernels (oplib/opcuda/sgemv3.cu, sgemv4.cu).
//
// Precision modes
//   OPB_FP32_PLAIN   : FP32 SIMT squaring and chaining exactly as the reference's FP32
//                      device path (no renormalisation).
//   OPB_FP32_RENORM  : the same with FP64 row renormalisation after every product.
//   OPB_FP16X3       : as OPB_BF16X3 with FP16 parts of 2^15-scaled values (11 + 11
//                      significant bits per split instead of 8 + 8; same cost).
//   OPB_BF16X3       : split-BF16 tensor-core products.  Squaring runs on E = U - I
//                      (E' = 2E + E.E, so the O(dt*L) information in U0 is not lost to
//                      BF16 rounding of entries near 1), FP64 row renormalisation after
//                      every product, chaining and pricing in split-BF16 as well.
// All launches go to the library stream without host synchronisation, so a whole solve
// can be captured in a CUDA graph.  The caller owns every buffer (workspace included),
// as with the reference's CArray buffers (oplib/opmodel/types/CArray.cs:550-590).
#include <cmath>

#include "common.cuh"
#include "lattice.h"

enum { OPB_FP32_PLAIN = 0, OPB_FP32_RENORM = 1, OPB_BF16X3 = 2, OPB_FP16X3 = 3 };

// FP16 parts: E-form and P-form entries are bounded by 1 in magnitude, so a 2^15 scale
// keeps them below the FP16 maximum with 11 + 11 significant bits.
constexpr float F16_SCALE = 32768.f;
inline bool tc_mode(int mode) { return mode == OPB_BF16X3 || mode == OPB_FP16X3; }

struct opb_lattice_desc {
    int d;                     // states
    int y0;                    // quoted state
    int ell_width;             // > 0: generator given as ELL (gen_cols, gen_vals); 0: dense gen_dense
    const int *gen_cols;       // device [d * ell_width], column index or -1
    const double *gen_vals;    // device [d * ell_width], FP64 rates
    const double *gen_dense;   // device [d * d] FP64, row-major (source-major)
    const double *x;           // device [d] spot value per state
    double dt;                 // elementary step: period * 2^-niter
    int niter;                 // squarings
    int nmat;                  // maturities T_m = m * period
    double period;
    double rate;               // continuously compounded discount rate
    int nK;                    // strikes
    const double *strikes;     // device [nK]
};

namespace {
int tc_gemm_ksplit(const opb::TcGemmArgs &a, cudaStream_t s);

struct Ws {
    // carve a workspace into 256-byte aligned pieces
    char *p;
    size_t used;
    template <class T>
    T *take(size_t n) {
        size_t off = (used + 255) & ~size_t(255);
        T *r = reinterpret_cast<T *>(p ? p + off : nullptr);
        used = off + n * sizeof(T);
        return r;
    }
};

struct Bufs {
    float *X, *Pa, *Pb, *G, *V, *gscale;
    __nv_bfloat16 *Ahi, *Alo, *Bhi, *Blo, *GThi, *GTlo;
    double *part;
    double2 *fix;  // per-row (s, inv) of the last E-form renormalisation (deferred into the next Cin)
    double *Vd;    // FP64 option values of the backward induction, d x nKp
    int *band;     // the ELL generator's half-bandwidth, found on the device per solve
    double *xpad;  // spot values of the padded lattice (split modes, d % 128 != 0)
};

inline int padded_nk(int nK, int mode) { return tc_mode(mode) ? (nK + 63) / 64 * 64 : nK; }

// The split modes run on multiples of 128 states: a lattice of another size is solved as one
// padded with absorbing states (zero generator rows and columns).  No state of the lattice
// reaches a padding state, so P(t) is block diagonal, [[P_lattice(t), 0], [0, I]], and the
// lattice's rows of every product, renormalisation and price are the unpadded ones.
inline int padded_d(int d, int mode) { return tc_mode(mode) ? (d + 127) / 128 * 128 : d; }

Bufs carve(Ws &w, int d, int nK, int mode, bool pad = false) {
    Bufs b{};
    size_t dd = (size_t)d * d;
    nK = padded_nk(nK, mode);
    b.X = w.take<float>(dd);
    b.Pa = w.take<float>(dd);
    if (!tc_mode(mode)) b.Pb = w.take<float>(dd);
    // the small-N products (pricing, induction) may run as up to 4 K-slices
    b.V = w.take<float>((size_t)d * nK * (tc_mode(mode) ? 4 : 1));
    b.gscale = w.take<float>(64);
    if (tc_mode(mode)) {
        b.Ahi = w.take<__nv_bfloat16>(dd);
        b.Alo = w.take<__nv_bfloat16>(dd);
        b.Bhi = w.take<__nv_bfloat16>(dd);
        b.Blo = w.take<__nv_bfloat16>(dd);
        b.GThi = w.take<__nv_bfloat16>((size_t)d * nK);
        b.GTlo = w.take<__nv_bfloat16>((size_t)d * nK);
        int np = opb::tc_gemm_nparts(d, d);
        b.part = w.take<double>((size_t)(np > 0 ? np : 1) * d);
        b.fix = w.take<double2>((size_t)d);
        b.Vd = w.take<double>((size_t)d * nK);
        b.band = w.take<int>(1);
        if (pad) b.xpad = w.take<double>((size_t)d);
    } else {
        b.G = w.take<float>((size_t)d * nK);
        b.part = w.take<double>((size_t)d);
        b.Vd = w.take<double>((size_t)d * nK);
    }
    return b;
}

#define LT(expr)                         \
    do {                                 \
        int _r = (expr);                 \
        if (_r != 0) return _r;          \
    } while (0)

// U0 = I + dt*L in FP32, niter FP32 squarings (with FP64 row renormalisation in
// OPB_FP32_RENORM) ping-ponging through X, Pa, Pb; *cur receives the index of P1.
int square_fp32(const opb_lattice_desc &L, int mode, Bufs &b, cudaStream_t s, int *cur_out) {
    const int d = L.d;
    // U0 in FP32 from FP64 arithmetic
    if (L.ell_width > 0) LT(opb::launch_ek_ell(d, L.ell_width, L.gen_cols, L.gen_vals, L.dt, 0, b.X, s));
    else LT(opb::launch_ek_dense(d, L.gen_dense, L.dt, 0, b.X, s));
    float *buf[3] = {b.X, b.Pa, b.Pb};
    int cur = 0, nxt = 1;
    for (int r = 0; r < L.niter; r++) {
        LT(opb::sgemm_rm(d, d, d, 1.f, buf[cur], d, buf[cur], d, 0.f, buf[nxt], d, s));
        if (mode == OPB_FP32_RENORM) {
            LT(opb::launch_rowsum(d, buf[nxt], b.part, s));
            LT(opb::launch_renorm(d, buf[nxt], b.part, 1, 0, nullptr, nullptr, nullptr, nullptr, s));
        }
        int t = cur; cur = nxt; nxt = t;
    }
    *cur_out = cur;
    return 0;
}

int solve_fp32(const opb_lattice_desc &L, int mode, Bufs &b, double *quotes, double *V_all, cudaStream_t s,
               float *P_out) {
    const int d = L.d, nK = L.nK;
    int cur = 0;
    LT(square_fp32(L, mode, b, s, &cur));
    float *buf[3] = {b.X, b.Pa, b.Pb};
    // buf[cur] = P(period); the chain alternates between the two other buffers
    float *P1 = buf[cur];
    if (P_out) return (int)cudaMemcpyAsync(P_out, P1, sizeof(float) * (size_t)d * d, cudaMemcpyDeviceToDevice, s);
    float *chain[2];
    for (int i = 0, k = 0; i < 3; i++)
        if (i != cur) chain[k++] = buf[i];
    LT(opb::launch_payoff(d, nK, nK, L.x, L.strikes, b.G, nullptr, nullptr, s));
    const float *Pm = P1;
    for (int m = 1; m <= L.nmat; m++) {
        if (m > 1) {
            float *out = chain[m & 1 ? 1 : 0];
            LT(opb::sgemm_rm(d, d, d, 1.f, Pm, d, P1, d, 0.f, out, d, s));
            if (mode == OPB_FP32_RENORM) {
                LT(opb::launch_rowsum(d, out, b.part, s));
                LT(opb::launch_renorm(d, out, b.part, 1, 0, nullptr, nullptr, nullptr, nullptr, s));
            }
            Pm = out;
        }
        LT(opb::sgemm_rm(d, nK, d, 1.f, Pm, d, b.G, nK, 0.f, b.V, nK, s));
        const double disc = std::exp(-L.rate * L.period * m);
        LT(opb::launch_discount(d, nK, nK, b.V, disc, V_all ? V_all + (size_t)(m - 1) * d * nK : nullptr, L.y0,
                                quotes + (size_t)(m - 1) * nK, s));
    }
    return 0;
}

// Issue every tensor-core product as S K-slices accumulated through the FP32 epilogue
// (C = slice + 1*C, round-to-nearest), which shortens each in-TMEM accumulation chain:
// the tensor cores truncate the FP32 accumulator, a bias of about half an ulp per MMA.
// 0 = automatic (one launch: the GEMM kernel already sums K in chunks of 2 K-blocks).
int g_ksplit = 0;

int tc_gemm_ksplit(const opb::TcGemmArgs &a, cudaStream_t s) {
    int S = g_ksplit > 0 ? g_ksplit : 1;
    int kb = a.K / 64;
    // (products that fuse their normalisation or splits into the epilogue run in one launch)
    if (S <= 1 || kb < S || kb % S || a.ksplit > 1 || a.band || a.Shi || a.fixmode >= opb::OPB_FIX_SQUARE)
        return opb::launch_tc_gemm(a, s);
    const int kslice = a.K / S;
    for (int i = 0; i < S; i++) {
        opb::TcGemmArgs t = a;
        t.K = kslice;
        t.Ahi = a.Ahi + (size_t)i * kslice;
        t.Alo = a.Alo + (size_t)i * kslice;
        const size_t boff = a.b_kn ? (size_t)i * kslice * a.ldb : (size_t)i * kslice;  // K rows or K columns
        t.Bhi = a.Bhi + boff;
        t.Blo = a.Blo + boff;
        if (i > 0) { t.Cin = a.C; t.beta = 1.f; t.cin_fix = nullptr; }
        if (i + 1 < S) t.rowsum = nullptr;
        int r = opb::launch_tc_gemm(t, s);
        if (r) return r;
    }
    return 0;
}

// E0 = dt*L, niter split squarings with renormalisation: P1 = P(period) as row-major splits
// in both the A and the B buffers and as FP32 in X.  g returns the product arguments of
// the squarings (B read K x N row-major), with B set to P1's B parts.
int square_tc(const opb_lattice_desc &L, Bufs &b, cudaStream_t s, bool f16, opb::TcGemmArgs &g, int d_gen) {
    const int d = L.d;
    const int np = opb::tc_gemm_nparts(d, d);
    const float ss = f16 ? F16_SCALE : 0.f;                    // split scale of E / P parts
    const float unscale = f16 ? 1.f / (F16_SCALE * F16_SCALE) : 1.f;
    // E0 = dt*L in FP32 (FP64 arithmetic), then its splits.  An ELL generator's band h0
    // bounds E_r's to h0 * 2^r: the squarings skip the K-blocks (and whole output tiles) that
    // only multiply zeros, with bit-identical results.
    // (d_gen < d: the generator's d_gen states, then absorbing padding states)
    if (d_gen != d) LT(opb::launch_ek_padded(d_gen, d, L.ell_width, L.gen_cols, L.gen_vals, L.gen_dense, L.dt, b.X, s));
    if (L.ell_width > 0) {
        if (d_gen == d) LT(opb::launch_ek_ell(d, L.ell_width, L.gen_cols, L.gen_vals, L.dt, 1, b.X, s));
        LT(opb::launch_ell_band(d_gen, L.ell_width, L.gen_cols, b.band, s));
    } else if (d_gen == d) {
        LT(opb::launch_ek_dense(d, L.gen_dense, L.dt, 1, b.X, s));
    }
    LT(opb::launch_split(d, d, b.X, d, b.Ahi, b.Alo, nullptr, nullptr, d, s, ss));
    // every squaring and chain product reads its B operand K x N row-major (MN-major):
    // a squaring's B is E's own row-major parts, a chain product's B the row-major parts of
    // P1 kept in the B buffers
    g = opb::TcGemmArgs{};
    g.M = d; g.N = d; g.K = d; g.lda = d; g.ldb = d; g.ldc = d; g.f16 = f16 ? 1 : 0; g.b_kn = 1;
    g.Ahi = b.Ahi; g.Alo = b.Alo; g.Bhi = b.Ahi; g.Blo = b.Alo;
    // The squarings write the next level's parts themselves, ping-ponging between the A and
    // the B part buffers; the normalisation of level r's output is deferred into level r + 1's
    // epilogue (OPB_FIX_SQUARE).  A level skips the output tiles that no K-block reaches,
    // so its part buffer must be zero there: A holds E0's parts (zero outside the band) and
    // B starts zeroed; the band only grows, so the tiles a level skips are zero in both.
    // (lattices not fused, opb::fused_single: a renormalisation kernel after every level,
    // which writes the next level's parts)
    const bool fused = opb::fused_single(d);
    if (fused && L.niter > 1) {
        LT((int)cudaMemsetAsync(b.Bhi, 0, sizeof(__nv_bfloat16) * (size_t)d * d, s));
        LT((int)cudaMemsetAsync(b.Blo, 0, sizeof(__nv_bfloat16) * (size_t)d * d, s));
    }
    __nv_bfloat16 *ph[2] = {b.Ahi, b.Bhi}, *pl[2] = {b.Alo, b.Blo};
    for (int r = 0; r < L.niter; r++) {
        // E' = 2E + E.E in place of E (X), with FP64 row-sum partials.  From the second level
        // on, X and the parts hold the previous level's output as its epilogue left it, and
        // that output's normalisation (b.fix, from its row sums) is applied in this epilogue.
        const bool last = r + 1 == L.niter;
        const int cur = fused ? (r & 1) : 0;
        g.Ahi = ph[cur]; g.Alo = pl[cur]; g.Bhi = ph[cur]; g.Blo = pl[cur];
        g.C = b.X; g.Cin = b.X; g.alpha = unscale; g.beta = 2.f; g.rowsum = b.part;
        g.cin_fix = r > 0 ? b.fix : nullptr;
        g.fixmode = r == 0 ? opb::OPB_FIX_NONE : fused ? opb::OPB_FIX_SQUARE : opb::OPB_FIX_CIN;
        g.Shi = (last || !fused) ? nullptr : ph[cur ^ 1];
        g.Slo = (last || !fused) ? nullptr : pl[cur ^ 1];
        g.sscale = ss;
        g.band = L.ell_width > 0 ? b.band : nullptr;
        g.band_skip = opb::g_band_skip;
        g.level = r;
        // BF16 parts: the lo.lo product on the first levels (see OPB_LOLO_LEVELS)
        g.lolo = (!f16 && r < opb::g_lolo_levels) ? 1 : 0;
        LT(tc_gemm_ksplit(g, s));
        // the last level emits P1 = I + E and its splits (row-major into A: the first
        // chain's A and pricing's; row-major into B: every chain's B); the others only the
        // row fixes of their output
        if (last) LT(opb::launch_renorm_to_p(d, b.X, b.part, np, b.Ahi, b.Alo, b.Bhi, b.Blo, s, ss));
        else if (fused) LT(opb::launch_rowfix(d, b.part, np, 1, b.fix, s));
        else LT(opb::launch_renorm(d, b.X, b.part, np, 1, b.Ahi, b.Alo, nullptr, nullptr, s, ss, 0, b.fix));
    }
    g.Ahi = b.Ahi; g.Alo = b.Alo;
    g.cin_fix = nullptr;
    g.fixmode = opb::OPB_FIX_NONE;
    g.Shi = g.Slo = nullptr;
    g.band = nullptr;
    g.band_skip = 0;
    g.level = 0;
    g.lolo = 0;
    if (L.niter == 0) {
        LT(opb::launch_add_identity(d, b.X, s));
        LT(opb::launch_split(d, d, b.X, d, b.Ahi, b.Alo, nullptr, nullptr, d, s, ss));
        LT(opb::launch_split(d, d, b.X, d, b.Bhi, b.Blo, nullptr, nullptr, d, s, ss));
    }
    g.Bhi = b.Bhi; g.Blo = b.Blo;
    return 0;
}

// d_gen: the lattice's own states (L.d when unpadded); V_all and P_out hold only those.
int solve_tc(const opb_lattice_desc &L, Bufs &b, double *quotes, double *V_all, cudaStream_t s, float *P_out,
             bool f16, int d_gen) {
    const int d = L.d, nK = L.nK;
    const int np = opb::tc_gemm_nparts(d, d);
    const float ss = f16 ? F16_SCALE : 0.f;                    // split scale of E / P parts
    const float unscale = f16 ? 1.f / (F16_SCALE * F16_SCALE) : 1.f;
    opb::TcGemmArgs g{};
    LT(square_tc(L, b, s, f16, g, d_gen));
    if (P_out)
        return (int)cudaMemcpy2DAsync(P_out, sizeof(float) * d_gen, b.X, sizeof(float) * d, sizeof(float) * d_gen, d_gen,
                                      cudaMemcpyDeviceToDevice, s);
    const int nKp = padded_nk(nK, OPB_BF16X3);
    const float *gs = nullptr;
    if (f16) {
        LT(opb::launch_payoff_scale(d, L.x, nK, L.strikes, b.gscale, s));
        gs = b.gscale;
    }
    LT(opb::launch_payoff(d, nK, nKp, L.x, L.strikes, nullptr, b.GThi, b.GTlo, s, gs));
    opb::TcGemmArgs pg{};
    pg.M = d; pg.N = nKp; pg.K = d; pg.lda = d; pg.ldb = d; pg.ldc = nKp; pg.f16 = g.f16;
    pg.Ahi = b.Ahi; pg.Alo = b.Alo; pg.Bhi = b.GThi; pg.Blo = b.GTlo; pg.C = b.V; pg.beta = 0.f;
    pg.alpha = f16 ? 1.f / F16_SCALE : 1.f;  // the payoff scale is undone in the FP64 discount
    // K-slices fill the GPU with this small-N product's tiles; the discount sums them
    pg.ksplit = opb::tc_gemm_split_for(d, nKp, d);
    pg.c_slice = (long long)d * nKp;
    // The chain products write only the parts of their output, ping-ponging between the A
    // part buffers and a second pair carved from the FP32 chain buffer (unused in the split
    // modes); each output's row normalisation is deferred into the next chain product's
    // epilogue and into its own pricing's discount (row scaling commutes with the products).
    // (lattices not fused: FP32 chain products renormalised by a kernel that writes the
    // parts into A, as the squarings are)
    const bool fused = opb::fused_single(d);
    const size_t dd = (size_t)d * d;
    __nv_bfloat16 *ch_hi[2] = {b.Ahi, reinterpret_cast<__nv_bfloat16 *>(b.Pa)};
    __nv_bfloat16 *ch_lo[2] = {b.Alo, reinterpret_cast<__nv_bfloat16 *>(b.Pa) + dd};
    int cur = 0;
    for (int m = 1; m <= L.nmat; m++) {
        if (m > 1 && fused) {
            // P_m = P_{m-1} . P1 (A: P_{m-1}'s parts, B: P1's), scaled by P_{m-1}'s row fix
            g.Ahi = ch_hi[cur]; g.Alo = ch_lo[cur];
            g.C = nullptr; g.Cin = nullptr; g.alpha = unscale; g.beta = 0.f; g.rowsum = b.part;
            g.cin_fix = m > 2 ? b.fix : nullptr;
            g.fixmode = m > 2 ? opb::OPB_FIX_ROWSCALE : opb::OPB_FIX_NONE;
            g.Shi = ch_hi[cur ^ 1]; g.Slo = ch_lo[cur ^ 1]; g.sscale = ss;
            LT(tc_gemm_ksplit(g, s));
            LT(opb::launch_rowfix(d, b.part, np, 0, b.fix, s));
            cur ^= 1;
        } else if (m > 1) {
            // P_m = P_{m-1} . P1 (A splits hold P_{m-1}, B splits P1), renormalise, split
            // row-major into A
            g.C = b.Pa; g.Cin = nullptr; g.alpha = unscale; g.beta = 0.f; g.rowsum = b.part;
            LT(tc_gemm_ksplit(g, s));
            LT(opb::launch_renorm(d, b.Pa, b.part, np, 0, b.Ahi, b.Alo, nullptr, nullptr, s, ss, 0));
        }
        pg.Ahi = ch_hi[cur]; pg.Alo = ch_lo[cur];
        LT(tc_gemm_ksplit(pg, s));
        const double disc = std::exp(-L.rate * L.period * m);
        LT(opb::launch_discount(d_gen, nK, nKp, b.V, disc, V_all ? V_all + (size_t)(m - 1) * d_gen * nK : nullptr,
                                L.y0, quotes + (size_t)(m - 1) * nK, s, gs, pg.ksplit, pg.c_slice,
                                (m > 1 && fused) ? b.fix : nullptr));
    }
    return 0;
}

// Backward induction on the period kernel: V_nmat = e(x), then for m = nmat-1 .. 0
// V_m = e^{-r period} P1 . V_{m+1}, knocked out below the barrier at the dates m >= 1 and,
// with exercise, floored by the exercise value there.  Each product runs on the tensor
// cores with V's split parts as a K x N row-major B operand.
int bermudan_tc(const opb_lattice_desc &L, Bufs &b, int put, int exercise, double barrier, double *quotes,
                cudaStream_t s, bool f16, int d_gen) {
    const int d = L.d, nK = L.nK, nKp = padded_nk(nK, OPB_BF16X3);
    opb::TcGemmArgs g{};
    LT(square_tc(L, b, s, f16, g, d_gen));
    const float *gs = nullptr;
    if (f16) {
        LT(opb::launch_berm_scale(d, L.x, nK, L.strikes, put, b.gscale, s));
        gs = b.gscale;
    }
    // V's parts live in the payoff-part buffers (d x nKp each)
    LT(opb::launch_berm_init(d, nK, nKp, L.x, L.strikes, put, barrier, b.Vd, b.GThi, b.GTlo, nullptr, gs, s));
    opb::TcGemmArgs pg{};
    pg.M = d; pg.N = nKp; pg.K = d; pg.lda = d; pg.ldb = nKp; pg.ldc = nKp; pg.f16 = f16 ? 1 : 0; pg.b_kn = 1;
    pg.Ahi = b.Ahi; pg.Alo = b.Alo; pg.Bhi = b.GThi; pg.Blo = b.GTlo; pg.C = b.V; pg.beta = 0.f;
    pg.alpha = f16 ? 1.f / F16_SCALE : 1.f;  // the P1 part scale; V's scale is undone in the step
    pg.ksplit = opb::tc_gemm_split_for(d, nKp, d);  // K-slices, summed by the step
    pg.c_slice = (long long)d * nKp;
    const double disc = std::exp(-L.rate * L.period);
    for (int m = L.nmat - 1; m >= 0; m--) {
        LT(tc_gemm_ksplit(pg, s));
        const bool last = m == 0;
        LT(opb::launch_berm_step(d, nK, nKp, b.V, disc, L.x, L.strikes, put, last ? 0.0 : barrier,
                                 last ? 0 : exercise, b.Vd, last ? nullptr : b.GThi, last ? nullptr : b.GTlo, nullptr,
                                 gs, L.y0, last ? quotes : nullptr, s, pg.ksplit, pg.c_slice));
    }
    return 0;
}

// The same induction with FP32 SIMT products (the reference's FP32 arithmetic; with
// OPB_FP32_RENORM the squarings are renormalised in FP64).
int bermudan_fp32(const opb_lattice_desc &L, int mode, Bufs &b, int put, int exercise, double barrier,
                  double *quotes, cudaStream_t s) {
    const int d = L.d, nK = L.nK;
    int cur = 0;
    LT(square_fp32(L, mode, b, s, &cur));
    float *buf[3] = {b.X, b.Pa, b.Pb};
    const float *P1 = buf[cur];
    LT(opb::launch_berm_init(d, nK, nK, L.x, L.strikes, put, barrier, b.Vd, nullptr, nullptr, b.G, nullptr, s));
    const double disc = std::exp(-L.rate * L.period);
    for (int m = L.nmat - 1; m >= 0; m--) {
        LT(opb::sgemm_rm(d, nK, d, 1.f, P1, d, b.G, nK, 0.f, b.V, nK, s));
        const bool last = m == 0;
        LT(opb::launch_berm_step(d, nK, nK, b.V, disc, L.x, L.strikes, put, last ? 0.0 : barrier,
                                 last ? 0 : exercise, b.Vd, nullptr, nullptr, last ? nullptr : b.G, nullptr, L.y0,
                                 last ? quotes : nullptr, s));
    }
    return 0;
}

int check_desc(const opb_lattice_desc *L, int mode) {
    if (!L) return OPB_E_NULL;
    if (L->d <= 0 || L->y0 < 0 || L->y0 >= L->d || L->niter < 0 || L->nmat < 1 || L->nK < 1) return OPB_E_ARG;
    if (!(L->dt > 0.0) || !(L->period > 0.0)) return OPB_E_ARG;
    if (!L->x || !L->strikes) return OPB_E_NULL;
    if (L->ell_width > 0) {
        if (!L->gen_cols || !L->gen_vals) return OPB_E_NULL;
    } else if (!L->gen_dense) {
        return OPB_E_NULL;
    }
    if (mode < OPB_FP32_PLAIN || mode > OPB_FP16X3) return OPB_E_ARG;
    if (tc_mode(mode) && opb::tc_gemm_tile_n(padded_d(L->d, mode)) == 0) return OPB_E_UNSUPPORTED;
    return OPB_OK;
}

// The lattice the split modes solve: L itself, or L padded with absorbing states (its spot
// values extended into b.xpad).
int prepare_padded(const opb_lattice_desc &L, int mode, Bufs &b, opb_lattice_desc &out, cudaStream_t s) {
    out = L;
    const int dp = padded_d(L.d, mode);
    if (dp == L.d) return 0;
    out.d = dp;
    out.x = b.xpad;
    return opb::launch_pad_x(L.d, dp, L.x, b.xpad, s);
}

}  // namespace

namespace opb {
int g_lolo_levels = OPB_LOLO_LEVELS;
int g_band_skip = 1;
int g_fused_max_d = -1;
}  // namespace opb

// Tuning knob: max_d >= 0 makes single-lattice solves of at most max_d states defer each
// product's row normalisation into the next product's epilogue, which also writes the next
// operand's parts (no renormalisation kernel between products), and larger ones renormalise
// with a kernel after every product (0: every size uses the kernel).  max_d = -1 restores
// the default: lattices of OPB_FUSED_AUTO_MIN_D states or more fuse, smaller ones use the
// kernel.
OPB_API int opb_set_fused_normalisation(int max_d) {
    OPB_REQUIRE(max_d >= -1, OPB_E_ARG);
    opb::g_fused_max_d = max_d;
    return opb::set_status(OPB_OK);
}

OPB_API int opb_set_lolo_levels(int n) {
    OPB_REQUIRE(n >= 0 && n <= 64, OPB_E_ARG);
    opb::g_lolo_levels = n;
    return opb::set_status(OPB_OK);
}

OPB_API int opb_set_band_skip(int on) {
    OPB_REQUIRE(on == 0 || on == 1, OPB_E_ARG);
    opb::g_band_skip = on;
    return opb::set_status(OPB_OK);
}

OPB_API int opb_set_ksplit(int s) {
    OPB_REQUIRE(s >= 0 && s <= 64, OPB_E_ARG);
    g_ksplit = s;
    return opb::set_status(OPB_OK);
}

// Workspace bytes for opb_lattice_solve.
OPB_API unsigned long long opb_lattice_workspace_size(int d, int nK, int mode) {
    if (d <= 0 || nK <= 0) return 0;
    Ws w{nullptr, 0};
    const int dp = padded_d(d, mode);
    (void)carve(w, dp, nK, mode, dp != d);
    return (unsigned long long)w.used + 256;
}

// Solves one lattice.  quotes: device [nmat * nK] FP64 (quotes[(m-1)*nK + k] is the
// price at state y0 of the call with strike k and maturity m*period).  V_all (optional):
// device [nmat * d * nK] FP64 prices at every state.  workspace: device, at least
// opb_lattice_workspace_size(d, nK, mode) bytes.
OPB_API int opb_lattice_solve(const opb_lattice_desc *L, int mode, void *workspace, unsigned long long ws_bytes,
                              double *quotes, double *V_all) {
    OPB_NVTX("opb_lattice_solve");
    int c = check_desc(L, mode);
    if (c == OPB_OK && !quotes) c = OPB_E_NULL;
    if (c != OPB_OK) return opb::set_status(c);
    OPB_REQUIRE(workspace, OPB_E_NULL);
    OPB_REQUIRE(ws_bytes >= opb_lattice_workspace_size(L->d, L->nK, mode), OPB_E_ARG);
    Ws w{reinterpret_cast<char *>(workspace), 0};
    size_t off = (256 - (reinterpret_cast<uintptr_t>(workspace) & 255)) & 255;
    w.p += off;
    const int dp = padded_d(L->d, mode);
    Bufs b = carve(w, dp, L->nK, mode, dp != L->d);
    cudaStream_t s = opb::stream();
    int r;
    if (tc_mode(mode)) {
        opb_lattice_desc Lp;
        r = prepare_padded(*L, mode, b, Lp, s);
        if (r == 0) r = solve_tc(Lp, b, quotes, V_all, s, nullptr, mode == OPB_FP16X3, L->d);
    } else {
        r = solve_fp32(*L, mode, b, quotes, V_all, s, nullptr);
    }
    return opb::set_status(r);
}

// Bermudan or barrier options on one lattice by backward induction on the period kernel
// P1 = P(period) (an extension: the reference ships the induction kernels, sgemv3/sgemv4,
// but no pricer on them).  Calls (put = 0) or puts (put = 1) with strikes L->strikes and
// final maturity T = nmat * period; exercise = 1: exercisable at T_m = m * period for m =
// 1..nmat (Bermudan), 0: at T only; barrier > 0: knocked out when the spot is at or below
// the barrier on any date T_m (m >= 1).  exercise = 0 with barrier = 0 gives the European
// value at T.  quotes: device [nK] FP64, the values at state y0.  In the split modes the
// induction products run on the tensor cores, in the FP32 modes on the SIMT GEMM;
// workspace as for opb_lattice_solve.
OPB_API int opb_lattice_bermudan(const opb_lattice_desc *L, int mode, int put, int exercise, double barrier,
                                 void *workspace, unsigned long long ws_bytes, double *quotes) {
    OPB_NVTX("opb_lattice_bermudan");
    int c = check_desc(L, mode);
    if (c == OPB_OK && !quotes) c = OPB_E_NULL;
    if (c == OPB_OK && (put < 0 || put > 1 || exercise < 0 || exercise > 1 || !(barrier >= 0.0))) c = OPB_E_ARG;
    if (c != OPB_OK) return opb::set_status(c);
    OPB_REQUIRE(workspace, OPB_E_NULL);
    OPB_REQUIRE(ws_bytes >= opb_lattice_workspace_size(L->d, L->nK, mode), OPB_E_ARG);
    Ws w{reinterpret_cast<char *>(workspace), 0};
    size_t off = (256 - (reinterpret_cast<uintptr_t>(workspace) & 255)) & 255;
    w.p += off;
    const int dp = padded_d(L->d, mode);
    Bufs b = carve(w, dp, L->nK, mode, dp != L->d);
    cudaStream_t s = opb::stream();
    if (!tc_mode(mode)) return opb::set_status(bermudan_fp32(*L, mode, b, put, exercise, barrier, quotes, s));
    opb_lattice_desc Lp;
    int r = prepare_padded(*L, mode, b, Lp, s);
    if (r == 0) r = bermudan_tc(Lp, b, put, exercise, barrier, quotes, s, mode == OPB_FP16X3, L->d);
    return opb::set_status(r);
}

// Transition kernel only: P_out (device, d x d FP32, source-major) = P(period) after
// niter squarings of U0 (no chaining, no pricing; nmat, nK and strikes are ignored).
OPB_API int opb_lattice_kernel(const opb_lattice_desc *L, int mode, void *workspace, unsigned long long ws_bytes,
                               float *P_out) {
    OPB_REQUIRE(L != nullptr, OPB_E_NULL);
    opb_lattice_desc L2 = *L;
    L2.nmat = 1;
    if (L2.nK < 1) L2.nK = 64;
    if (!L2.strikes) L2.strikes = reinterpret_cast<const double *>(L2.x);
    int c = check_desc(&L2, mode);
    if (c != OPB_OK) return opb::set_status(c);
    OPB_REQUIRE(workspace && P_out, OPB_E_NULL);
    OPB_REQUIRE(ws_bytes >= opb_lattice_workspace_size(L2.d, L2.nK, mode), OPB_E_ARG);
    Ws w{reinterpret_cast<char *>(workspace), 0};
    size_t off = (256 - (reinterpret_cast<uintptr_t>(workspace) & 255)) & 255;
    w.p += off;
    const int dp = padded_d(L2.d, mode);
    Bufs b = carve(w, dp, L2.nK, mode, dp != L2.d);
    cudaStream_t s = opb::stream();
    int r;
    if (tc_mode(mode)) {
        opb_lattice_desc Lp;
        r = prepare_padded(L2, mode, b, Lp, s);
        if (r == 0) r = solve_tc(Lp, b, nullptr, nullptr, s, P_out, mode == OPB_FP16X3, L2.d);
    } else {
        r = solve_fp32(L2, mode, b, nullptr, nullptr, s, P_out);
    }
    return opb::set_status(r);
}

// Step kernels of a Monte Carlo plan whose steps span several elementary intervals (a
// generator date inside a step): the kernel of such a step is the product of its elementary
// kernels in time order.  The reference plans the factor lists (jfactor_ms,
// oplib/opmodel/models/CModel Common.cs:431-486) and chains them on the device with FP32
// products (device_mc_sminit / smk / smcopy, CModel Device.cs:252-295); here each product is
// an FP32 GEMM followed by the FP64 row renormalisation of the lattice solve.  factors: host
// array of nf device pointers to row-major (source-major) d x d FP32 kernels; out must not
// alias them.  workspace: opb_chain_workspace_size(d) bytes.
OPB_API unsigned long long opb_chain_workspace_size(int d) {
    if (d <= 0) return 0;
    Ws w{nullptr, 0};
    (void)w.take<float>((size_t)d * d);
    (void)w.take<double>((size_t)d);
    return (unsigned long long)w.used + 256;
}

OPB_API int opb_chain_kernels(int d, int nf, const float *const *factors, float *out, void *workspace,
                              unsigned long long ws_bytes) {
    OPB_NVTX("opb_chain_kernels");
    OPB_REQUIRE(d > 0 && nf >= 1, OPB_E_ARG);
    OPB_REQUIRE(factors && out, OPB_E_NULL);
    for (int i = 0; i < nf; i++) {
        OPB_REQUIRE(factors[i] != nullptr, OPB_E_NULL);
        OPB_REQUIRE(factors[i] != out, OPB_E_ARG);
    }
    cudaStream_t s = opb::stream();
    const size_t bytes = sizeof(float) * (size_t)d * d;
    if (nf == 1) return opb::set_status((int)cudaMemcpyAsync(out, factors[0], bytes, cudaMemcpyDeviceToDevice, s));
    OPB_REQUIRE(workspace, OPB_E_NULL);
    OPB_REQUIRE(ws_bytes >= opb_chain_workspace_size(d), OPB_E_ARG);
    Ws w{reinterpret_cast<char *>(workspace), 0};
    w.p += (256 - (reinterpret_cast<uintptr_t>(workspace) & 255)) & 255;
    float *tmp = w.take<float>((size_t)d * d);
    double *part = w.take<double>((size_t)d);
    // the products alternate between out and tmp so that the last one lands in out
    const float *cur = factors[0];
    for (int i = 1; i < nf; i++) {
        float *dst = ((nf - 1 - i) % 2 == 0) ? out : tmp;
        int r = opb::sgemm_rm(d, d, d, 1.f, cur, d, factors[i], d, 0.f, dst, d, s);
        if (r == 0) r = opb::launch_rowsum(d, dst, part, s);
        if (r == 0) r = opb::launch_renorm(d, dst, part, 1, 0, nullptr, nullptr, nullptr, nullptr, s);
        if (r != 0) return opb::set_status(r);
        cur = dst;
    }
    return opb::set_status(OPB_OK);
}

// The reference's plan rule for one interval (oplib/opmodel/models/CModel Common.cs:289-307):
// dt = min(0.5 / maxdiag, dt0), niter = ceil(log2(DeltaT / dt)), dt_j = DeltaT * 2^-niter.
OPB_API int opb_plan_interval(double maxdiag, double delta_t, double dt0, int *niter, double *dt_j) {
    OPB_REQUIRE(niter && dt_j, OPB_E_NULL);
    OPB_REQUIRE(delta_t > 0.0 && dt0 > 0.0 && maxdiag >= 0.0, OPB_E_ARG);
    double dt = maxdiag > 0.0 ? 0.5 / maxdiag : dt0;
    if (dt > dt0) dt = dt0;
    int n = (int)std::ceil(std::log(delta_t / dt) / std::log(2.0));
    *niter = n;
    *dt_j = delta_t * std::pow(2.0, -n);
    return opb::set_status(OPB_OK);
}
