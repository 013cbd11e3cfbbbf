// Generator builders on the device, in FP64, emitting the sparse (ELL) form consumed by
// the lattice solve.
//
// Local volatility (width 3, columns y-1, y, y+1): per interior node the down/up rates
// solve [dm dp; dm^2 dp^2] p = [drift, vol^2] with dm = x[y-1]-x[y], dp = x[y+1]-x[y]
// (oplib/opmodel/types/S1DGrid.cs:78-147 builds the 2x2 inverses,
// oplib/opmodel/models/CLVModel.cs:86-136 applies them); boundary nodes are absorbing;
// the diagonal is minus the row sum.
//
// Stochastic volatility (width 7): spot x log-spaced (nx), variance V = sigma_v^2 with
// sigma_v log-spaced (nv), state y = ix + nx*iv (oplib/opmodel/types/S2DGrid.cs:142).
// Heston variance dynamics dV = kappa(theta - V)dt + xi sqrt(V) dW2 with spot-variance
// correlation rho, carried by two diagonal moves at a common rate q capped so that they
// never carry more variance than the target in either direction; axial rates from the
// per-direction 2x2 moment systems (the block-diagonal 4x4 invm of S2DGrid.pregen,
// S2DGrid.cs:123-245); negative rates clamped to zero and a spot drift fix-up to r*x
// (oplib/opmodel/models/CSVModel.cs:331-376).  The correlation term is a project
// extension: the reference's SV generator has none.
#include <cstring>

#include "common.cuh"
#include "lattice.h"

namespace opb {

// The moment-matching solve of one interior node: rates pm (down) and pp (up) with
// pm dm + pp dp = a and pm dm^2 + pp dp^2 = b.  Every operation is rounded explicitly
// (no contraction into FMAs), so all kernels that build LV rows agree bit for bit.
__device__ __forceinline__ void lv_rates(double dm, double dp, double a, double b, double &pm, double &pp) {
    const double det = __dsub_rn(__dmul_rn(__dmul_rn(dm, dp), dp), __dmul_rn(__dmul_rn(dp, dm), dm));
    pm = __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn(dp, dp), a), __dmul_rn(dp, b)), det);
    pp = __ddiv_rn(__dadd_rn(__dmul_rn(__dmul_rn(-dm, dm), a), __dmul_rn(dm, b)), det);
}

// sigma(x) = max(floor, level + skew*exp(-((x-1)/width)^2)), explicitly rounded.
__device__ __forceinline__ double lv_sigma_at(double xv, double level, double skew, double width, double floor_) {
    const double z = __ddiv_rn(__dsub_rn(xv, 1.0), width);
    double sg = __dadd_rn(level, __dmul_rn(skew, exp(-__dmul_rn(z, z))));
    return sg > floor_ ? sg : floor_;
}

// x_i = s0*lo*(hi/lo)^(i/(n-1)).
__device__ __forceinline__ double lv_node(int n, double lo, double hi, double s0, int y) {
    return __dmul_rn(__dmul_rn(s0, lo), pow(__ddiv_rn(hi, lo), __ddiv_rn((double)y, (double)(n - 1))));
}

__global__ void k_lv_ell(int d, const double *__restrict__ x, const double *__restrict__ drift,
                         const double *__restrict__ vol, int *__restrict__ cols, double *__restrict__ vals) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= d) return;
    double pm = 0.0, pp = 0.0;
    if (y > 0 && y < d - 1) {
        const double dm = __dsub_rn(x[y - 1], x[y]), dp = __dsub_rn(x[y + 1], x[y]);
        const double v = vol[y];
        lv_rates(dm, dp, drift[y], __dmul_rn(v, v), pm, pp);
    }
    int *c = cols + 3LL * y;
    double *v = vals + 3LL * y;
    c[0] = y > 0 ? y - 1 : -1;
    v[0] = y > 0 ? pm : 0.0;
    c[1] = y;
    v[1] = -((y > 0 ? pm : 0.0) + (y < d - 1 ? pp : 0.0));
    c[2] = y < d - 1 ? y + 1 : -1;
    v[2] = y < d - 1 ? pp : 0.0;
}

// sigma(x) = max(floor, level + skew*exp(-((x-1)/width)^2)); x_i = lo*(hi/lo)^(i/(n-1));
// drift = r*x, vol = sigma(x)*x.  Writes x, drift and vol.
__global__ void k_lv_params(int d, double lo, double hi, double s0, double level, double skew, double width,
                            double floor_, double r, double *__restrict__ x, double *__restrict__ drift,
                            double *__restrict__ vol) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= d) return;
    const double xv = lv_node(d, lo, hi, s0, y);
    x[y] = xv;
    drift[y] = __dmul_rn(r, xv);
    vol[y] = __dmul_rn(lv_sigma_at(xv, level, skew, width, floor_), xv);
}

// Many LV lattices in one launch (calibration loops): thread per global row; lattice i
// owns rows row_off .. row_off + n - 1 of the concatenated ELL arrays.  The arithmetic is
// k_lv_params followed by k_lv_ell, node by node, so the entries are bit-identical.
struct LvParam {
    int n, pad;
    long long row_off;
    double level, skew, width, floor_, rate;
};

__global__ void k_lv_ell_batched(int nlat, const LvParam *__restrict__ P, long long total_rows, double lo, double hi,
                                 double s0, int *__restrict__ cols, double *__restrict__ vals) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= total_rows) return;
    int a = 0, b = nlat - 1;
    while (a < b) {  // last lattice with row_off <= g
        const int mid = (a + b + 1) >> 1;
        if (P[mid].row_off <= g) a = mid; else b = mid - 1;
    }
    const LvParam p = P[a];
    const int d = p.n, y = (int)(g - p.row_off);
    double pm = 0.0, pp = 0.0;
    if (y > 0 && y < d - 1) {
        const double xv = lv_node(d, lo, hi, s0, y);
        const double v = __dmul_rn(lv_sigma_at(xv, p.level, p.skew, p.width, p.floor_), xv);
        const double dm = __dsub_rn(lv_node(d, lo, hi, s0, y - 1), xv);
        const double dp = __dsub_rn(lv_node(d, lo, hi, s0, y + 1), xv);
        lv_rates(dm, dp, __dmul_rn(p.rate, xv), __dmul_rn(v, v), pm, pp);
    }
    int *c = cols + 3LL * g;
    double *v = vals + 3LL * g;
    c[0] = y > 0 ? y - 1 : -1;
    v[0] = y > 0 ? pm : 0.0;
    c[1] = y;
    v[1] = -((y > 0 ? pm : 0.0) + (y < d - 1 ? pp : 0.0));
    c[2] = y < d - 1 ? y + 1 : -1;
    v[2] = y < d - 1 ? pp : 0.0;
}

// The reference's two-dimensional generator with jumps across volatility levels (the
// drop-in for oplib/opcuda/sgsvg.cu:40-236).  Thread per (interval i, source y0); the row
// of y0 in interval i is built in place in the dense column-major FP32 output
// (element y0 -> y1 at gen[i*d*d + y0 + d*y1]); arithmetic in FP64, entries stored in FP32:
//   1. neighbour rates invm . (0, svol^2 [interior x], voldrift, volvol^2 [interior r]);
//   2. for r1 > r0 with prob = sum of the row's level-r1 entries > 0: entries x1 < x0-1 and
//      x1 > x0 of level r1 become prob * w / sum(w), w = exp(+-(x1 - x0) / (J x0)) with
//      J = jump size below / above (the reference kernel reads the lower size for both,
//      sgsvg.cu:111-112; the host model uses each side's own, CSVModel.cs:301-312);
//   3. negative off-diagonal entries cleared, the drift corrected through one neighbour
//      with the reference's formula (sgsvg.cu:166-207), diagonal = -(off-diagonal sum).
// par: x [d], then sdrift, svol, voldrift, volvol, jump_minus, jump_plus, each [ni][d].
__global__ void k_sgsvg(float *__restrict__ gen, int ni, int nx, int nr, const float *__restrict__ invm,
                        const float *__restrict__ par) {
    const int d = nx * nr;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)ni * d) return;
    const int i = (int)(t / d), y0 = (int)(t - (long long)i * d);
    const int r0 = y0 / nx, x0 = y0 - r0 * nx;
    const float *xv = par;
    const long long pi = (long long)d + (long long)i * d + y0;
    const long long pstride = (long long)ni * d;
    // blocks after x: sdrift, svol, voldrift, volvol, jump_minus, jump_plus (sgsvg.cu:223-229)
    const double sdrift = par[pi], sv = par[pi + pstride], vd = par[pi + 2 * pstride], vv = par[pi + 3 * pstride];
    const double jmin0 = par[pi + 4 * pstride], jplus0 = par[pi + 5 * pstride];
    float *g = gen + (long long)i * d * d + y0;  // row y0: g[d * y1]
    const double xo = xv[y0];
    double rhs[4] = {0.0, (x0 > 0 && x0 < nx - 1) ? sv * sv : 0.0, vd, (r0 > 0 && r0 < nr - 1) ? vv * vv : 0.0};
    double q[4];
    for (int k = 0; k < 4; k++) {
        double acc = 0.0;
        for (int j = 0; j < 4; j++) acc += (double)invm[16LL * y0 + k + 4 * j] * rhs[j];
        q[k] = acc;
    }
    if (x0 > 0) g[(long long)d * (y0 - 1)] = (float)q[0];
    if (x0 < nx - 1) g[(long long)d * (y0 + 1)] = (float)q[1];
    if (r0 > 0) g[(long long)d * (y0 - nx)] = (float)q[2];
    if (r0 < nr - 1) g[(long long)d * (y0 + nx)] = (float)q[3];
    // jumps to higher volatility levels
    const double jmin = jmin0 * xo, jplus = jplus0 * xo;
    for (int r1 = r0 + 1; r1 < nr; r1++) {
        const int base = nx * r1;
        double prob = 0.0;
        for (int x1 = 0; x1 < nx; x1++) prob += (double)g[(long long)d * (base + x1)];
        if (!(prob > 0.0)) continue;
        double sum0 = 0.0;
        if (jmin > 0.0)
            for (int x1 = 0; x1 < x0 - 1; x1++) sum0 += exp(((double)xv[base + x1] - xo) / jmin);
        if (jplus > 0.0)
            for (int x1 = x0 + 1; x1 < nx; x1++) sum0 += exp(-((double)xv[base + x1] - xo) / jplus);
        if (!(sum0 > 0.0)) continue;
        const double ratio = prob / sum0;
        if (jmin > 0.0)
            for (int x1 = 0; x1 < x0 - 1; x1++)
                g[(long long)d * (base + x1)] = (float)(ratio * exp(((double)xv[base + x1] - xo) / jmin));
        if (jplus > 0.0)
            for (int x1 = x0 + 1; x1 < nx; x1++)
                g[(long long)d * (base + x1)] = (float)(ratio * exp(-((double)xv[base + x1] - xo) / jplus));
    }
    // sum rules: clear negatives, correct the drift, conserve probability
    double drift = 0.0, tot = 0.0;
    for (int y1 = 0; y1 < d; y1++) {
        if (y1 == y0) continue;
        float *e = g + (long long)d * y1;
        const double v = *e;
        if (v < 0.0) {
            *e = 0.f;
        } else {
            drift += v * ((double)xv[y1] - xo);
            tot += v;
        }
    }
    if (drift > sdrift) {
        if (x0 > 0) {
            const double ratio = (drift - sdrift) / ((double)xv[y0 - 1] - xo);
            float *e = g + (long long)d * (y0 - 1);
            *e = (float)((double)*e + ratio);
            tot += ratio;
        }
    } else if (x0 < nx - 1) {
        const double ratio = (sdrift - drift) / ((double)xv[y0 + 1] - xo);
        float *e = g + (long long)d * (y0 + 1);
        *e = (float)((double)*e + ratio);
        tot += ratio;
    }
    g[(long long)d * y0] = (float)(-tot);
}

struct SvArgs {
    int nx, nv;
    double x_lo, x_hi, v_lo, v_hi, r, kappa, theta, xi, rho;
};

__device__ __forceinline__ double sv_xs(const SvArgs &a, int ix) {
    return a.x_lo * pow(a.x_hi / a.x_lo, (double)ix / (double)(a.nx - 1));
}
__device__ __forceinline__ double sv_V(const SvArgs &a, int iv) {
    double s = a.v_lo * pow(a.v_hi / a.v_lo, (double)iv / (double)(a.nv - 1));
    return s * s;
}

__global__ void k_sv_ell(SvArgs a, int *__restrict__ cols, double *__restrict__ vals, double *__restrict__ x_y) {
    const int d = a.nx * a.nv;
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= d) return;
    const int ix = y % a.nx, iv = y / a.nx;
    int c[7];
    double v[7];
    for (int j = 0; j < 7; j++) { c[j] = -1; v[j] = 0.0; }
    const double x = sv_xs(a, ix);
    if (x_y) x_y[y] = x;
    c[6] = y;
    if (ix == 0 || ix == a.nx - 1) {  // absorbing spot boundary
        cols[7LL * y + 0] = y; vals[7LL * y + 0] = 0.0;
        for (int j = 1; j < 7; j++) { cols[7LL * y + j] = -1; vals[7LL * y + j] = 0.0; }
        return;
    }
    const double V = sv_V(a, iv);
    const double var_x = V * x * x, var_v = a.xi * a.xi * V, cov = a.rho * a.xi * V * x;
    const double mu_x = a.r * x, mu_v = a.kappa * (a.theta - V);
    const double xm = sv_xs(a, ix - 1), xp = sv_xs(a, ix + 1);
    const double dxm = xm - x, dxp = xp - x;
    // slots: 0 x-1, 1 x+1, 2 v-1, 3 v+1, 4 diag A, 5 diag B, 6 self
    c[0] = y - 1; c[1] = y + 1;
    double q = 0.0, ex = 0.0, ev = 0.0, ex2 = 0.0, ev2 = 0.0;
    double dxa = 0, dva = 0, dxb = 0, dvb = 0;
    if (iv > 0 && iv < a.nv - 1 && a.rho != 0.0) {
        const double dvm = sv_V(a, iv - 1) - V, dvp = sv_V(a, iv + 1) - V;
        if (a.rho < 0.0) {
            dxa = dxp; dva = dvm; c[4] = (ix + 1) + a.nx * (iv - 1);
            dxb = dxm; dvb = dvp; c[5] = (ix - 1) + a.nx * (iv + 1);
        } else {
            dxa = dxp; dva = dvp; c[4] = (ix + 1) + a.nx * (iv + 1);
            dxb = dxm; dvb = dvm; c[5] = (ix - 1) + a.nx * (iv - 1);
        }
        const double cx = dxa * dva + dxb * dvb;
        const double sx2 = dxa * dxa + dxb * dxb, sv2 = dva * dva + dvb * dvb;
        q = cov / cx;
        q = fmin(q, var_x / sx2);
        q = fmin(q, var_v / sv2);
        q = fmax(q, 0.0);
        v[4] = q; v[5] = q;
        ex = q * (dxa + dxb); ev = q * (dva + dvb); ex2 = q * sx2; ev2 = q * sv2;
    }
    {
        const double aa = mu_x - ex, bb = var_x - ex2;
        const double det = dxm * dxp * dxp - dxp * dxm * dxm;
        v[0] = (dxp * dxp * aa - dxp * bb) / det;
        v[1] = (-dxm * dxm * aa + dxm * bb) / det;
    }
    if (iv > 0 && iv < a.nv - 1) {
        const double dvm = sv_V(a, iv - 1) - V, dvp = sv_V(a, iv + 1) - V;
        const double aa = mu_v - ev, bb = var_v - ev2;
        const double det = dvm * dvp * dvp - dvp * dvm * dvm;
        c[2] = y - a.nx; v[2] = (dvp * dvp * aa - dvp * bb) / det;
        c[3] = y + a.nx; v[3] = (-dvm * dvm * aa + dvm * bb) / det;
    } else if (iv == 0) {
        c[3] = y + a.nx; v[3] = fmax(mu_v, 0.0) / (sv_V(a, 1) - V);
    } else {
        c[2] = y - a.nx; v[2] = fmin(mu_v, 0.0) / (sv_V(a, iv - 1) - V);
    }
    // clamp, drift of the clamped stencil, fix-up
    double drift = 0.0;
    for (int j = 0; j < 6; j++) {
        if (c[j] < 0) continue;
        if (v[j] < 0.0) v[j] = 0.0;
        const int tx = c[j] % a.nx;
        const double dxj = (tx == ix) ? 0.0 : (tx == ix - 1 ? dxm : dxp);
        drift += v[j] * dxj;
    }
    if (drift > mu_x) v[0] += (drift - mu_x) / (x - xm);
    else v[1] += (mu_x - drift) / (xp - x);
    double tot = 0.0;
    for (int j = 0; j < 6; j++)
        if (c[j] >= 0) tot += v[j];
    v[6] = -tot;
    for (int j = 0; j < 7; j++) {
        cols[7LL * y + j] = c[j];
        vals[7LL * y + j] = c[j] >= 0 ? v[j] : 0.0;
    }
}

// max over rows of |L_yy| for an ELL generator (column == row entry).
__global__ void k_maxdiag(int d, int w, const int *__restrict__ cols, const double *__restrict__ vals,
                          unsigned long long *__restrict__ out_bits) {
    double m = 0.0;
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < d; y += gridDim.x * blockDim.x)
        for (int j = 0; j < w; j++)
            if (cols[(long long)y * w + j] == y) m = fmax(m, fabs(vals[(long long)y * w + j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));  // m >= 0
}

}  // namespace opb

using namespace opb;

OPB_API int opb_lv_params(int d, double lo, double hi, double s0, double level, double skew, double width,
                          double floor_, double r, double *x, double *drift, double *vol) {
    OPB_REQUIRE(d >= 3, OPB_E_ARG);
    OPB_REQUIRE(x && drift && vol, OPB_E_NULL);
    OPB_REQUIRE(lo > 0.0 && hi > lo && width > 0.0, OPB_E_ARG);
    k_lv_params<<<(d + 255) / 256, 256, 0, stream()>>>(d, lo, hi, s0, level, skew, width, floor_, r, x, drift, vol);
    return launch_check();
}

// LV generator in ELL form (width 3) from per-node spot values, drifts and vols.
OPB_API int opb_lv_generator_ell(int d, const double *x, const double *drift, const double *vol, int *cols,
                                 double *vals) {
    OPB_REQUIRE(d >= 3, OPB_E_ARG);
    OPB_REQUIRE(x && drift && vol && cols && vals, OPB_E_NULL);
    k_lv_ell<<<(d + 255) / 256, 256, 0, stream()>>>(d, x, drift, vol, cols, vals);
    return launch_check();
}

// LV generators of nlat lattices in one launch, into concatenated ELL arrays (width 3).
// params: device array of nlat records {int n, pad; int64 row_off; double level, skew,
// width, floor, rate} (56 bytes), row_off ascending from 0; total_rows = sum of n.
OPB_API int opb_lv_generator_ell_batched(int nlat, const void *params, long long total_rows, double lo, double hi,
                                         double s0, int *cols, double *vals) {
    OPB_REQUIRE(nlat > 0 && total_rows >= 3 && lo > 0.0 && hi > lo && s0 > 0.0, OPB_E_ARG);
    OPB_REQUIRE(params && cols && vals, OPB_E_NULL);
    OPB_REQUIRE(aligned(params, 8), OPB_E_ALIGN);
    const long long g = (total_rows + 255) / 256;
    k_lv_ell_batched<<<(unsigned)g, 256, 0, stream()>>>(nlat, reinterpret_cast<const LvParam *>(params), total_rows,
                                                      lo, hi, s0, cols, vals);
    return launch_check();
}

OPB_API int opb_lv_param_size(void) { return (int)sizeof(LvParam); }

// Drop-in for opcuda_sgsvg (oplib/opcuda/sgsvg.cu:215-236), 64-bit handles: ni intervals of
// the dense column-major FP32 generator of an nx x nr grid from the per-node moment
// inverses invmat [16 d] and the parameter block par (see k_sgsvg).  The caller zeroes
// gen first, as the reference's caller does.
OPB_API int opcuda_sgsvg(unsigned long long gen_yyi_ptr, int ni, int nx, int nr, unsigned long long invmat_ptr,
                         unsigned long long parptr) {
    OPB_REQUIRE(ni > 0 && nx >= 2 && nr >= 2, OPB_E_ARG);
    OPB_REQUIRE(gen_yyi_ptr && invmat_ptr && parptr, OPB_E_NULL);
    const long long n = (long long)ni * nx * nr;
    k_sgsvg<<<(unsigned)((n + 127) / 128), 128, 0, stream()>>>(
        reinterpret_cast<float *>(gen_yyi_ptr), ni, nx, nr, reinterpret_cast<const float *>(invmat_ptr),
        reinterpret_cast<const float *>(parptr));
    return launch_check();
}

// SV generator in ELL form (width 7); x_y (optional) receives the spot value per state.
OPB_API int opb_sv_generator_ell(int nx, int nv, double x_lo, double x_hi, double v_lo, double v_hi, double r,
                                 double kappa, double theta, double xi, double rho, int *cols, double *vals,
                                 double *x_y) {
    OPB_REQUIRE(nx >= 3 && nv >= 3, OPB_E_ARG);
    OPB_REQUIRE(x_lo > 0.0 && x_hi > x_lo && v_lo > 0.0 && v_hi > v_lo && xi >= 0.0, OPB_E_ARG);
    OPB_REQUIRE(rho > -1.0 && rho < 1.0, OPB_E_ARG);
    OPB_REQUIRE(cols && vals, OPB_E_NULL);
    SvArgs a{nx, nv, x_lo, x_hi, v_lo, v_hi, r, kappa, theta, xi, rho};
    int d = nx * nv;
    k_sv_ell<<<(d + 127) / 128, 128, 0, stream()>>>(a, cols, vals, x_y);
    return launch_check();
}

// max |L_yy| (blocking: the value is returned to the host for the squaring plan).
// dscratch: one device word (8 bytes) owned by the caller.
OPB_API int opb_ell_maxdiag(int d, int w, const int *cols, const double *vals, unsigned long long *dscratch,
                            double *out_host) {
    OPB_REQUIRE(d > 0 && w > 0, OPB_E_ARG);
    OPB_REQUIRE(cols && vals && dscratch && out_host, OPB_E_NULL);
    OPB_TRY(cudaMemsetAsync(dscratch, 0, sizeof(unsigned long long), stream()));
    int g = (d + 255) / 256;
    k_maxdiag<<<g < 1024 ? g : 1024, 256, 0, stream()>>>(d, w, cols, vals, dscratch);
    unsigned long long bits = 0;
    OPB_TRY(cudaMemcpyAsync(&bits, dscratch, sizeof(bits), cudaMemcpyDeviceToHost, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    double v;
    std::memcpy(&v, &bits, sizeof(v));
    *out_host = v;
    return set_status(OPB_OK);
}
