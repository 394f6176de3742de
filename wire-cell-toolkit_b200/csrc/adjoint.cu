// Adjoint (reverse-mode derivative) of the DepoTransform forward path.
//
// Forward (kernels.cu), per plane:
//   Q_g[w][t]  = sum over depo patches of qn * t_tau * (a_k or b_k)      (raster)
//   F[o][t]    = sum_g sum_j (R_g[j] (x) Q_g[o - npad - j])[t]          (FFT convolution)
// with, per patch bin k of a depo (pitch) and tau (time),
//   p_k = Phi(u_{k+1}) - Phi(u_k),  u = (edge - c_p) / sigma_p
//   a_k = p_k * w_k = [sigma_p (phi(u_{k+1}) - phi(u_k)) + (e_{k+1} - c_p) p_k] / bs
//   b_k = p_k - a_k,   t_tau likewise in time,   qn = q' / (sum p * sum t)
// (GaussianDiffusion.cxx:30-92,116-182; BinnedDiffusion_transform.cxx:296-367).
//
// Backward, per plane, given G = dL/dF on the frame window:
//   dQ_g[i] = sum_j conj(R_g[j]) * G[i + npad + j]   (per frequency; transposed convolution)
//   then per depo: gather the patch cells of dQ and apply the closed-form
//   derivatives of p, a, t and qn, chained through the drift
//   (Drifter.cxx:164-192) to (t, q, x, y, z, extent_long, extent_tran) and to
//   the global DL, DT and lifetime.  Patch windows are recomputed (k_prep_all),
//   never stored, and treated as fixed (the window edges are the only
//   non-differentiable points of the model).

#include "gauss.cuh"
#include "kernels.cuh"

namespace wctb200 {

// ---------------------------------------------------------------------------
// dL/dF of one plane as real grid rows: row o is wire wire0 + o, column c is
// tick tick0 + c; zero outside the reference window and the readout.
// ---------------------------------------------------------------------------
__global__ void k_grad_rows(const float* __restrict__ gframe, int nticks, int wire0, int wlo, int whi, int tick0,
                            int ncols, int nrows, int N, float* __restrict__ out)
{
    const int o = blockIdx.y;
    const int W = wire0 + o;
    const bool wok = W >= wlo && W < whi;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int t = tick0 + c;
        float v = 0.f;
        if (wok && c < ncols && t >= 0 && t < nticks) v = gframe[(size_t)W * nticks + t];
        out[(size_t)o * N + c] = v;
    }
}

void launch_grad_rows(const float* gframe, int nticks, int wire0, int wlo, int whi, int tick0, int ncols, int nrows,
                      int N, float* out, cudaStream_t s)
{
    if (nrows <= 0) return;
    dim3 grid((N + 255) / 256, nrows);
    k_grad_rows<<<grid, 256, 0, s>>>(gframe, nticks, wire0, wlo, whi, tick0, ncols, nrows, N, out);
}

// ---------------------------------------------------------------------------
// Transposed wire convolution in the (wire, frequency) domain:
//   dQ_g[i][f] = sum_{j=-P}^{P} conj(R_g[j][f]) * G[i + P + j][f],  i in [0, nin)
// Block: 32 frequencies x 8 row groups, 8 consecutive rows per thread, the
// needed G rows staged in shared memory once for all groups.
// ---------------------------------------------------------------------------
constexpr int kAdjRB = 8;
constexpr int kAdjRG = 8;
constexpr int kAdjRows = kAdjRB * kAdjRG;

__global__ void __launch_bounds__(32 * kAdjRG) k_wire_conv_adj(const float2* __restrict__ Gh,
                                                                const float2* __restrict__ Rh,
                                                                float2* __restrict__ dQh, int G, int PAD, int nin,
                                                                int nout, int M)
{
    extern __shared__ float2 adj_smem[];
    const int SROWS = kAdjRows + 2 * PAD;
    const int NT = 2 * PAD + 1;
    float2(*Gs)[32] = reinterpret_cast<float2(*)[32]>(adj_smem);
    float2(*Rs)[32] = reinterpret_cast<float2(*)[32]>(adj_smem + (size_t)SROWS * 32);
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int f = blockIdx.x * 32 + lane;
    const int i0 = blockIdx.y * kAdjRows;
    const bool fok = f < M;
    const bool dc = f == 0;
    // rows i0 + s of G, s in [0, SROWS): input row i uses G rows i .. i + 2P
    for (int s = rg; s < SROWS; s += kAdjRG) {
        const int o = i0 + s;
        Gs[s][lane] = (fok && o < nout) ? Gh[(size_t)o * M + f] : make_float2(0.f, 0.f);
    }
    const int rb0 = rg * kAdjRB;
    for (int g = 0; g < G; ++g) {
        __syncthreads();
        for (int jj = rg; jj < NT; jj += kAdjRG)
            Rs[jj][lane] = fok ? Rh[((size_t)g * NT + jj) * M + f] : make_float2(0.f, 0.f);
        __syncthreads();
        if (!fok) continue;
        float2 acc[kAdjRB];
#pragma unroll
        for (int r = 0; r < kAdjRB; ++r) acc[r] = make_float2(0.f, 0.f);
        for (int jj = 0; jj < NT; ++jj) {
            const float2 rr = Rs[jj][lane];
            // conj(R) * G, component-wise in bin 0
            const float rc = dc ? 0.f : rr.y;
            const float ry = dc ? rr.y : rr.x;
#pragma unroll
            for (int r = 0; r < kAdjRB; ++r) {
                const float2 q = Gs[rb0 + r + jj][lane];
                acc[r].x = fmaf(rr.x, q.x, fmaf(rc, q.y, acc[r].x));
                acc[r].y = fmaf(ry, q.y, fmaf(-rc, q.x, acc[r].y));
            }
        }
#pragma unroll
        for (int r = 0; r < kAdjRB; ++r) {
            const int i = i0 + rb0 + r;
            if (i < nin) dQh[((size_t)g * nin + i) * M + f] = acc[r];
        }
    }
}

void launch_wire_conv_adj(const float2* Gh, const float2* Rh, float2* dQh, int G, int npad, int nin, int nout, int M,
                          cudaStream_t s)
{
    if (nin <= 0) return;
    dim3 grid((M + 31) / 32, (nin + kAdjRows - 1) / kAdjRows);
    dim3 block(32, kAdjRG);
    const size_t smem = sizeof(float2) * 32 * ((size_t)(kAdjRows + 2 * npad) + (2 * npad + 1));
    cudaFuncSetAttribute((const void*)k_wire_conv_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_wire_conv_adj<<<grid, block, smem, s>>>(Gh, Rh, dQh, G, npad, nin, nout, M);
}

// ---------------------------------------------------------------------------
// Per (plane, depo): gather the patch cells of dL/dQ and form the gradients.
// One warp per depo-plane: lanes over ticks, a loop over the impact bins,
// which are tabulated in shared memory in chunks of kGatherChunk bins.
//
// With x_k = edge_k - c (c the pitch centre, k = 0..np), u_k = x_k / s,
// phi the unit normal density and bs the impact bin size:
//   p_k      = Phi(u_{k+1}) - Phi(u_k)
//   a_k      = [s (phi(u_{k+1}) - phi(u_k)) + x_{k+1} p_k] / bs   (p_k * weight_k)
//   dp/dc    = -(phi_{k+1} - phi_k) / s
//   dp/ds    = -(u_{k+1} phi_{k+1} - u_k phi_k) / s
//   da/dc    = [(u phi)_{k+1} - (u phi)_k - p_k + x_{k+1} dp/dc] / bs
//   da/ds    = [phi_{k+1} - phi_k + (u^2 phi)_{k+1} - (u^2 phi)_k + x_{k+1} dp/ds] / bs
// and the same bin integrals and derivatives in time.  The patch adds
// qn t_tau a_k to group l and qn t_tau (p_k - a_k) to group l + 1 of its wire,
// qn = q / (sum_k p_k * sum_tau t_tau) (sums over the clipped patch).
// ---------------------------------------------------------------------------
constexpr int kGatherWarps = 4;
constexpr int kGatherChunk = 256;  // impact bins tabulated at once

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Derivatives of the unit bin integral between edges at distances x1 < x2
// from the centre, for sigma s > 0: returns p; dc, ds receive dp/dc, dp/ds.
__device__ __forceinline__ float bin_and_derivs(float x1, float x2, float s, float inv, float& dc, float& ds)
{
    const float u1 = x1 / s, u2 = x2 / s;
    const float f1 = norm_pdf(u1), f2 = norm_pdf(u2);
    dc = -(f2 - f1) / s;
    ds = -(u2 * f2 - u1 * f1) / s;
    const float e1 = copysignf(erfc_nr(fabsf(x1 * inv)), x1), e2 = copysignf(erfc_nr(fabsf(x2 * inv)), x2);
    return bin_from_edges(e1, e2);
}

__global__ void __launch_bounds__(kGatherWarps * 32) k_adj_gather(const double* __restrict__ dep, int n, DriftDev dd,
                                                                  int do_drift, PlaneSet ps, AdjSet as,
                                                                  double drift_speed,
                                                                  const PatchRec* __restrict__ rec,
                                                                  const float* __restrict__ dQ,
                                                                  double* __restrict__ grad,
                                                                  double* __restrict__ gglob)
{
    __shared__ float s_bin[kGatherWarps][kGatherChunk][6];  // a, p, da/dc, dp/dc, da/ds, dp/ds
    __shared__ double s_glob[kGatherWarps][3];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * kGatherWarps + wib;
    const long long total = (long long)ps.nplanes * n;
    double gDL = 0.0, gDT = 0.0, gTau = 0.0;
    if (gw < total) {
        const int ip = (int)(gw / n), i = (int)(gw - (long long)ip * n);
        const PatchRec r = rec[(size_t)ip * n + i];
        const AdjPlane& A = as.p[ip];
        const int np = r.np, nt = r.nt;
        if (np > 0 && nt > 0 && A.nin > 0) {
            const float pbs = A.pbs, tbs = A.tbs;
            const float sp = r.sp, st = r.st;
            const float invp = sp > 0.f ? 1.0f / (1.41421356237309505f * sp) : 0.f;
            const float invt = st > 0.f ? 1.0f / (1.41421356237309505f * st) : 0.f;
            // normalisation sums over the clipped patch and their derivatives
            float Sp = 1.f, dSp_c = 0.f, dSp_s = 0.f;
            if (sp > 0.f) Sp = bin_and_derivs(-r.pcr, (float)np * pbs - r.pcr, sp, invp, dSp_c, dSp_s);
            float St = 1.f, dSt_c = 0.f, dSt_s = 0.f;
            if (st > 0.f) St = bin_and_derivs(-r.tcr, (float)nt * tbs - r.tcr, st, invt, dSt_c, dSt_s);
            double acc_qn = 0.0, acc_cp = 0.0, acc_sp = 0.0, acc_ct = 0.0, acc_st = 0.0;
            const int nimp = A.nimp;
            const size_t gstride = (size_t)A.nin * A.N;
            for (int k0 = 0; k0 < np; k0 += kGatherChunk) {
                const int nk = min(kGatherChunk, np - k0);
                __syncwarp();
                for (int kk = lane; kk < nk; kk += 32) {
                    const int k = k0 + kk;
                    float a, p, dadc, dpdc, dads, dpds;
                    if (sp > 0.f) {
                        const float x1 = (float)k * pbs - r.pcr, x2 = (float)(k + 1) * pbs - r.pcr;
                        p = bin_and_derivs(x1, x2, sp, invp, dpdc, dpds);
                        const float u1 = x1 / sp, u2 = x2 / sp;
                        const float f1 = norm_pdf(u1), f2 = norm_pdf(u2);
                        a = (sp * (f2 - f1) + x2 * p) / pbs;
                        dadc = ((u2 * f2 - u1 * f1) - p + x2 * dpdc) / pbs;
                        dads = ((f2 - f1) + (u2 * u2 * f2 - u1 * u1 * f1) + x2 * dpds) / pbs;
                    }
                    else {  // point in pitch: one bin, weight (edge_{k+1} - c) / bs
                        p = 1.f;
                        a = (pbs - r.pcr) / pbs;
                        dpdc = dpds = dads = 0.f;
                        dadc = -1.0f / pbs;
                    }
                    float* sb = s_bin[wib][kk];
                    sb[0] = a;
                    sb[1] = p;
                    sb[2] = dadc;
                    sb[3] = dpdc;
                    sb[4] = dads;
                    sb[5] = dpds;
                }
                __syncwarp();
                for (int tc = 0; tc < nt; tc += 32) {
                    const int tau = tc + lane;
                    const bool on = tau < nt;
                    float tv = 0.f, dtc = 0.f, dts = 0.f;
                    if (on) {
                        if (st > 0.f)
                            tv = bin_and_derivs((float)tau * tbs - r.tcr, (float)(tau + 1) * tbs - r.tcr, st, invt, dtc,
                                                dts);
                        else tv = 1.f;
                    }
                    float U = 0.f, ac = 0.f, as_ = 0.f;
                    const int col = r.toff + tau - A.col0;
                    int kabs = r.poff + k0;
                    int wire = kabs / nimp;
                    int l = kabs - wire * nimp;
                    for (int kk = 0; kk < nk; ++kk) {
                        float D0 = 0.f, D1 = 0.f;
                        if (on) {
                            const float* b0 = dQ + A.qoff + ((size_t)l * A.nin + (wire - A.start_ch)) * A.N + col;
                            D0 = __ldg(b0);
                            D1 = __ldg(b0 + gstride);
                        }
                        const float* sb = s_bin[wib][kk];
                        const float a = sb[0], p = sb[1];
                        const float dd0 = D0 - D1;
                        U = fmaf(a, dd0, fmaf(p, D1, U));
                        ac = fmaf(dd0, sb[2], fmaf(D1, sb[3], ac));
                        as_ = fmaf(dd0, sb[4], fmaf(D1, sb[5], as_));
                        if (++l == nimp) {
                            l = 0;
                            ++wire;
                        }
                    }
                    acc_qn += (double)(tv * U);
                    acc_cp += (double)(tv * ac);
                    acc_sp += (double)(tv * as_);
                    acc_ct += (double)(U * dtc);
                    acc_st += (double)(U * dts);
                }
            }
            acc_qn = warp_sum_d(acc_qn);
            acc_cp = warp_sum_d(acc_cp);
            acc_sp = warp_sum_d(acc_sp);
            acc_ct = warp_sum_d(acc_ct);
            acc_st = warp_sum_d(acc_st);
            if (lane == 0) {
                const double qn = r.qn;
                const double gqn = acc_qn;
                // centres and widths, through qn = q / (Sp * St) as well
                const double gcp = qn * acc_cp - gqn * (qn / Sp) * dSp_c;
                const double gsp = qn * acc_sp - gqn * (qn / Sp) * dSp_s;
                const double gct = qn * acc_ct - gqn * (qn / St) * dSt_c;
                const double gst = qn * acc_st - gqn * (qn / St) * dSt_s;
                const double gqf = gqn / ((double)Sp * (double)St);
                const double gsL = gst / drift_speed;  // sigma_time = extent_long / drift_speed
                const double gsT = gsp;                // sigma_pitch = extent_tran
                // back through the drift (Drifter::insert, gen/src/Drifter.cxx:164-192)
                const double* pd = dep + 7 * (size_t)i;
                const double q0 = pd[1], x0 = pd[2], el0 = pd[5], et0 = pd[6];
                double gq = gqf, gx = 0.0, gel = gsL, get = gsT;
                if (do_drift) {
                    int found = -1;
                    double dir = 0.0;
                    for (int k = 0; k < dd.nxr; ++k) {
                        const double a = dd.xr[k][0], rp = dd.xr[k][1];
                        if ((a < x0 && x0 < rp) || (rp < x0 && x0 < a)) { found = k; dir = -1.0; break; }
                    }
                    if (found < 0)
                        for (int k = 0; k < dd.nxr; ++k) {
                            const double rp = dd.xr[k][1], c = dd.xr[k][2];
                            if ((rp < x0 && x0 < c) || (c < x0 && x0 < rp)) { found = k; dir = 1.0; break; }
                        }
                    if (found >= 0) {
                        const double respx = dd.xr[found][1];
                        const double dt = fabs((respx - x0) / dd.speed);
                        const double dtdx = (x0 > respx ? 1.0 : -1.0) / dd.speed;  // d(dt)/dx
                        if (dir > 0) {
                            // t' = t + dt, q' = q exp(-dt/lifetime), sL^2 = 2 DL dt + el^2, sT^2 = 2 DT dt + et^2
                            const double ex = exp(-dt / dd.lifetime);
                            const double qd = q0 * ex;
                            const double sL = sqrt(2.0 * dd.DL * dt + el0 * el0);
                            const double sT = sqrt(2.0 * dd.DT * dt + et0 * et0);
                            const double hL = sL > 0.0 ? gsL / sL : 0.0;  // dL/d(sL^2) * 2
                            const double hT = sT > 0.0 ? gsT / sT : 0.0;
                            const double gdt = gct - gqf * qd / dd.lifetime + hL * dd.DL + hT * dd.DT;
                            gx = gdt * dtdx;
                            gq = gqf * ex;
                            gel = hL * el0;
                            get = hT * et0;
                            gDL = hL * dt;
                            gDT = hT * dt;
                            gTau = gqf * qd * dt / (dd.lifetime * dd.lifetime);
                        }
                        else {
                            gx = -gct * dtdx;  // t' = t - dt in the response region
                        }
                    }
                }
                else {
                    gx = gcp * A.ax;
                }
                double* gd = grad + 7 * (size_t)i;
                atomicAdd(gd + 0, gct);
                atomicAdd(gd + 1, gq);
                atomicAdd(gd + 2, gx);
                atomicAdd(gd + 3, gcp * A.ay);
                atomicAdd(gd + 4, gcp * A.az);
                atomicAdd(gd + 5, gel);
                atomicAdd(gd + 6, get);
                (void)q0;
            }
        }
    }
    if (lane == 0) {
        s_glob[wib][0] = gDL;
        s_glob[wib][1] = gDT;
        s_glob[wib][2] = gTau;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int k = 0; k < kGatherWarps; ++k) v += s_glob[k][threadIdx.x];
        if (v != 0.0) atomicAdd(gglob + threadIdx.x, v);
    }
}

void launch_adj_gather(const double* depos, int n, const DriftDev& dd, int do_drift, const PlaneSet& ps,
                       const AdjSet& as, double drift_speed, const PatchRec* rec, const float* dQ, double* grad,
                       double* gglob, cudaStream_t s)
{
    const long long warps = (long long)ps.nplanes * n;
    if (warps <= 0) return;
    const long long blocks = (warps + kGatherWarps - 1) / kGatherWarps;
    k_adj_gather<<<(unsigned)blocks, kGatherWarps * 32, 0, s>>>(depos, n, dd, do_drift, ps, as, drift_speed, rec, dQ,
                                                                grad, gglob);
}

}  // namespace wctb200
