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
// Block: 32 frequencies x 8 row groups, 8 consecutive rows per thread with a
// register window over the G rows staged in shared memory once for all
// groups; the taps of group g + 1 are copied by cp.async into the second of
// two tap buffers while group g is multiplied out of the first.
// ---------------------------------------------------------------------------
constexpr int kAdjRB = 8;
constexpr int kAdjRG = 8;
constexpr int kAdjRows = kAdjRB * kAdjRG;

__global__ void __launch_bounds__(32 * kAdjRG) k_wire_conv_adj(const float2* __restrict__ Gh,
                                                                const float2* __restrict__ Rh,
                                                                float2* __restrict__ dQh, int G, int PAD, int nin,
                                                                int nout, int M)
{
    extern __shared__ __align__(16) float2 adj_smem[];
    const int SROWS = kAdjRows + 2 * PAD;
    const int NT = 2 * PAD + 1;
    float2(*Gs)[32] = reinterpret_cast<float2(*)[32]>(adj_smem);
    float2* Rbuf = adj_smem + (size_t)SROWS * 32;  // two tap buffers of NT x 32
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int tid = rg * 32 + lane;
    const int f0 = blockIdx.x * 32;
    const int f = f0 + lane;
    const int i0 = blockIdx.y * kAdjRows;
    const bool fok = f < M;
    const bool dc = f == 0;
    // taps of group g into buffer st: 16 pieces of 16 bytes per 32-frequency row (M even)
    auto issue = [&](int g, int st) {
        float2* Rs = Rbuf + (size_t)st * NT * 32;
        const int fp = f0 + 2 * (tid & 15);
        const int nb = fp < M ? 16 : 0;
        for (int e = tid; e < NT * 16; e += 32 * kAdjRG) {
            const int jj = e >> 4;
            cp_async16(Rs + jj * 32 + 2 * (e & 15), nb ? Rh + ((size_t)g * NT + jj) * M + fp : Rh, nb);
        }
        cp_async_commit();
    };
    issue(0, 0);
    // rows i0 + s of G, s in [0, SROWS): input row i uses G rows i .. i + 2P
    for (int s = rg; s < SROWS; s += kAdjRG) {
        const int o = i0 + s;
        Gs[s][lane] = (fok && o < nout) ? Gh[(size_t)o * M + f] : make_float2(0.f, 0.f);
    }
    const int rb0 = rg * kAdjRB;
    for (int g = 0; g < G; ++g) {
        if (g + 1 < G) {
            issue(g + 1, (g + 1) & 1);
            cp_async_wait<1>();
        }
        else
            cp_async_wait<0>();
        __syncthreads();  // group g's taps (and, at g = 0, the G rows) visible to every thread
        const float2* Rs = Rbuf + (size_t)(g & 1) * NT * 32;
        if (fok) {
            float2 acc[kAdjRB], win[kAdjRB];
#pragma unroll
            for (int r = 0; r < kAdjRB; ++r) {
                acc[r] = make_float2(0.f, 0.f);
                win[r] = Gs[rb0 + r][lane];
            }
            for (int jj = 0; jj < NT; ++jj) {
                const float2 rr = Rs[jj * 32 + lane];
                // conj(R) * G, component-wise in bin 0
                const float rc = dc ? 0.f : rr.y;
                const float ry = dc ? rr.y : rr.x;
#pragma unroll
                for (int r = 0; r < kAdjRB; ++r) {
                    const float2 q = win[r];  // G row rb0 + r + jj
                    acc[r].x = fmaf(rr.x, q.x, fmaf(rc, q.y, acc[r].x));
                    acc[r].y = fmaf(ry, q.y, fmaf(-rc, q.x, acc[r].y));
                }
#pragma unroll
                for (int r = 0; r < kAdjRB - 1; ++r) win[r] = win[r + 1];
                win[kAdjRB - 1] = Gs[min(rb0 + kAdjRB + jj, SROWS - 1)][lane];
            }
#pragma unroll
            for (int r = 0; r < kAdjRB; ++r) {
                const int i = i0 + rb0 + r;
                if (i < nin) dQh[((size_t)g * nin + i) * M + f] = acc[r];
            }
        }
        __syncthreads();  // buffer g & 1 is refilled with group g + 2 next
    }
}

void launch_wire_conv_adj(const float2* Gh, const float2* Rh, float2* dQh, int G, int npad, int nin, int nout, int M,
                          cudaStream_t s)
{
    if (nin <= 0) return;
    dim3 grid((M + 31) / 32, (nin + kAdjRows - 1) / kAdjRows);
    dim3 block(32, kAdjRG);
    const size_t smem = sizeof(float2) * 32 * ((size_t)(kAdjRows + 2 * npad) + 2 * (size_t)(2 * npad + 1));
    cudaFuncSetAttribute((const void*)k_wire_conv_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_wire_conv_adj<<<grid, block, smem, s>>>(Gh, Rh, dQh, G, npad, nin, nout, M);
}

// ---------------------------------------------------------------------------
// Per depo: gather the patch cells of dL/dQ on every plane and form the
// gradients.  One warp per depo; the patch is tabulated in shared memory in
// chunks (impact bins x ticks) and the chunk's cells are spread over the 32
// lanes, so every lane is busy whatever the patch shape.
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
// qn = q / (sum_k p_k * sum_tau t_tau) (sums over the clipped patch).  Every
// accumulated quantity is a sum over cells (k, tau) of a bin factor times a
// tick factor times dL/dQ, e.g. dL/dqn = sum tv_tau (a_k D0 + (p_k - a_k) D1).
// ---------------------------------------------------------------------------
constexpr int kGatherWarps = 4;
constexpr int kChunkP = 128;  // impact bins per table chunk
constexpr int kChunkT = 128;  // ticks per table chunk
constexpr int kUnroll = 4;    // cells per lane with loads in flight together

struct __align__(16) BinTab {
    float a, p, dadc, dpdc;
    float dads, dpds;
    int base;  // offset of (group l, charge row) of this bin in the plane grid, plus the patch's first column
    int pad;
};

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Quantities of one bin edge at distance x from the centre (sigma s > 0,
// is = 1/s, inv = 1/(sqrt(2) s)): the signed erfc of the forward's bin
// integrals, the density phi(u), u phi(u) and u^2 phi(u) with u = x/s.
__device__ __forceinline__ void edge_terms(float x, float is, float inv, float& E, float& f, float& uf, float& uuf)
{
    const float u = x * is;
    E = copysignf(erfc_nr(fabsf(x * inv)), x);
    f = norm_pdf(u);
    uf = u * f;
    uuf = u * uf;
}

__device__ __forceinline__ float warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kGatherWarps * 32, 5) k_adj_gather(int n, PlaneSet ps, AdjSet as, double inv_vd,
                                                                     const PatchRec* __restrict__ rec,
                                                                     const float* __restrict__ dQ,
                                                                     double* __restrict__ grad,
                                                                     const double* __restrict__ qscale)
{
    __shared__ BinTab s_p[kGatherWarps][kChunkP];
    __shared__ float4 s_t[kGatherWarps][kChunkT];
    const unsigned full = 0xffffffffu;
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kGatherWarps + wib;
    if (i >= n) return;  // whole warps only: no block-level barrier follows
    // per-depo sums over planes: dL/dt', dL/dq', dL/dsL, dL/dsT, dL/d(x', y, z) through the pitch
    double s_ct = 0.0, s_qf = 0.0, s_sL = 0.0, s_sT = 0.0, s_px = 0.0, s_py = 0.0, s_pz = 0.0;
    bool any = false;
    for (int ip = 0; ip < ps.nplanes; ++ip) {
        const PatchRec r = rec[(size_t)ip * n + i];
        const AdjPlane& A = as.p[ip];
        const int np = r.np, nt = r.nt;
        if (np == 0 || nt == 0 || A.nin == 0) continue;
        any = true;
        const float pbs = A.pbs, tbs = A.tbs, ipbs = 1.0f / pbs;
        const float sp = r.sp, st = r.st;
        const float isp = sp > 0.f ? 1.0f / sp : 0.f, invp = 0.70710678118654752f * isp;
        const float ist = st > 0.f ? 1.0f / st : 0.f, invt = 0.70710678118654752f * ist;
        // lane partial sums of the bin integrals and their derivatives (normalisation)
        float pS = 0.f, pSc = 0.f, pSs = 0.f, tS = 0.f, tSc = 0.f, tSs = 0.f;
        double acc_qn = 0.0, acc_cp = 0.0, acc_sp = 0.0, acc_ct = 0.0, acc_st = 0.0;
        const size_t gstride = (size_t)A.nin * A.N;
        const float* dQp = dQ + A.qoff;
        const int col = r.toff - A.col0;
        for (int t0 = 0; t0 < nt; t0 += kChunkT) {
            const int ntc = min(kChunkT, nt - t0);
            __syncwarp();
            if (st > 0.f) {
                // one edge per lane, bins from neighbouring lanes (31 bins per round)
                for (int tb = t0; tb < t0 + ntc; tb += 31) {
                    const int e = tb + lane;
                    const float x = (float)e * tbs - r.tcr;
                    float E = 0.f, f = 0.f, uf = 0.f, uuf = 0.f;
                    if (e <= nt) edge_terms(x, ist, invt, E, f, uf, uuf);
                    const float E2 = __shfl_down_sync(full, E, 1), f2 = __shfl_down_sync(full, f, 1);
                    const float uf2 = __shfl_down_sync(full, uf, 1);
                    if (lane < 31 && e < t0 + ntc) {
                        const float tv = bin_from_edges(E, E2);
                        const float dtc = -(f2 - f) * ist, dts = -(uf2 - uf) * ist;
                        s_t[wib][e - t0] = make_float4(tv, dtc, dts, 0.f);
                        tS += tv;
                        tSc += dtc;
                        tSs += dts;
                    }
                    (void)uuf;
                }
            }
            else if (lane == 0) {  // point in time: one tick
                s_t[wib][0] = make_float4(1.f, 0.f, 0.f, 0.f);
                tS = 1.f;
            }
            for (int k0 = 0; k0 < np; k0 += kChunkP) {
                const int nk = min(kChunkP, np - k0);
                __syncwarp();
                for (int kb = k0; kb < k0 + nk; kb += 31) {
                    const int e = kb + lane;
                    float E = 0.f, f = 0.f, uf = 0.f, uuf = 0.f;
                    if (sp > 0.f && e <= np) edge_terms((float)e * pbs - r.pcr, isp, invp, E, f, uf, uuf);
                    const float E2 = __shfl_down_sync(full, E, 1), f2 = __shfl_down_sync(full, f, 1);
                    const float uf2 = __shfl_down_sync(full, uf, 1), uuf2 = __shfl_down_sync(full, uuf, 1);
                    if (lane < 31 && e < k0 + nk) {
                        BinTab b;
                        if (sp > 0.f) {
                            const float x2 = (float)(e + 1) * pbs - r.pcr;
                            b.p = bin_from_edges(E, E2);
                            b.dpdc = -(f2 - f) * isp;
                            b.dpds = -(uf2 - uf) * isp;
                            b.a = fmaf(sp, f2 - f, x2 * b.p) * ipbs;
                            b.dadc = (((uf2 - uf) - b.p) + x2 * b.dpdc) * ipbs;
                            b.dads = (((f2 - f) + (uuf2 - uuf)) + x2 * b.dpds) * ipbs;
                        }
                        else {  // point in pitch: one bin, weight (edge_{k+1} - c) / bs
                            b.p = 1.f;
                            b.a = (pbs - r.pcr) * ipbs;
                            b.dpdc = b.dpds = b.dads = 0.f;
                            b.dadc = -ipbs;
                        }
                        const int kabs = r.poff + e;
                        const int wire = kabs / A.nimp;
                        const int l = kabs - wire * A.nimp;
                        b.base = (l * A.nin + (wire - A.start_ch)) * A.N + col + t0;
                        b.pad = 0;
                        s_p[wib][e - k0] = b;
                        if (t0 == 0) {
                            pS += b.p;
                            pSc += b.dpdc;
                            pSs += b.dpds;
                        }
                    }
                }
                __syncwarp();
                // cells c = lane + 32 m of the nk x ntc chunk, (k, tau) advanced
                // incrementally; kUnroll cells per lane have their loads in flight at once
                const int ncell = nk * ntc;
                const int dk = 32 / ntc, dt = 32 - dk * ntc;
                int k = lane / ntc, tau = lane - k * ntc;
                for (int c0 = 0; c0 < ncell; c0 += 32 * kUnroll) {
                    float D0[kUnroll], D1[kUnroll];
                    int kk[kUnroll], tt[kUnroll];
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) {
                        kk[u] = min(k, nk - 1);
                        tt[u] = tau;
                        D0[u] = D1[u] = 0.f;
                        if (c0 + lane + 32 * u < ncell) {
                            const float* q = dQp + s_p[wib][k].base + tau;
                            D0[u] = __ldg(q);
                            D1[u] = __ldg(q + gstride);
                        }
                        tau += dt;
                        k += dk;
                        if (tau >= ntc) {
                            tau -= ntc;
                            ++k;
                        }
                    }
                    // cells past the end loaded zeros and add nothing
                    float pq = 0.f, pc = 0.f, pss = 0.f, pct = 0.f, pst = 0.f;
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) {
                        const BinTab b = s_p[wib][kk[u]];
                        const float4 tq = s_t[wib][tt[u]];
                        const float dd0 = D0[u] - D1[u];
                        const float uu = fmaf(b.a, dd0, b.p * D1[u]);
                        const float vc = fmaf(b.dadc, dd0, b.dpdc * D1[u]);
                        const float vs = fmaf(b.dads, dd0, b.dpds * D1[u]);
                        pq = fmaf(tq.x, uu, pq);
                        pc = fmaf(tq.x, vc, pc);
                        pss = fmaf(tq.x, vs, pss);
                        pct = fmaf(tq.y, uu, pct);
                        pst = fmaf(tq.z, uu, pst);
                    }
                    acc_qn += (double)pq;
                    acc_cp += (double)pc;
                    acc_sp += (double)pss;
                    acc_ct += (double)pct;
                    acc_st += (double)pst;
                }
            }
        }
        // normalisation sums (whole warp), then this lane's share of the gradients:
        // every term is linear in the lane's partial sums, so the warp reduction
        // waits until all planes are done
        const float Sp = warp_sum_f(pS), dSp_c = warp_sum_f(pSc), dSp_s = warp_sum_f(pSs);
        const float St = warp_sum_f(tS), dSt_c = warp_sum_f(tSc), dSt_s = warp_sum_f(tSs);
        const float iSp = 1.0f / Sp, iSt = 1.0f / St;
        const double qn = r.qn;
        // centres and widths, through qn = q / (Sp * St) as well
        const double gcp = qn * acc_cp - acc_qn * (double)(r.qn * iSp * dSp_c);
        s_sT += qn * acc_sp - acc_qn * (double)(r.qn * iSp * dSp_s);                  // sigma_pitch = extent_tran
        s_ct += qn * acc_ct - acc_qn * (double)(r.qn * iSt * dSt_c);
        s_sL += (qn * acc_st - acc_qn * (double)(r.qn * iSt * dSt_s)) * inv_vd;      // sigma_time = extent_long / v
        // the plane's charge is qscale * q' (modify_depo): its share of dL/dq' carries the scale
        s_qf += acc_qn * (double)(iSp * iSt) * (qscale ? qscale[(size_t)i * ps.nplanes + ip] : 1.0);
        s_px += gcp * A.ax;
        s_py += gcp * A.ay;
        s_pz += gcp * A.az;
    }
    if (!any) return;
    s_ct = warp_sum_d(s_ct);
    s_qf = warp_sum_d(s_qf);
    s_px = warp_sum_d(s_px);
    s_py = warp_sum_d(s_py);
    s_pz = warp_sum_d(s_pz);
    s_sL = warp_sum_d(s_sL);
    s_sT = warp_sum_d(s_sT);
    if (lane == 0) {
        // sums over planes; k_adj_drift takes them back through the drift in place
        double* gd = grad + 7 * (size_t)i;
        gd[0] = s_ct;
        gd[1] = s_qf;
        gd[2] = s_px;
        gd[3] = s_py;
        gd[4] = s_pz;
        gd[5] = s_sL;
        gd[6] = s_sT;
    }
}

// Back through the drift (Drifter::insert, gen/src/Drifter.cxx:164-192), one
// thread per depo, in place on the per-depo sums of k_adj_gather
// (dL/dt', dL/dq', dL/d(x', y, z) through the pitch, dL/dsigma_L, dL/dsigma_T),
// plus the block sums of dL/d(DL, DT, lifetime).
__global__ void __launch_bounds__(256) k_adj_drift(const double* __restrict__ dep, int n, DriftDev dd,
                                                    double* __restrict__ grad, double* __restrict__ gglob)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double gDL = 0.0, gDT = 0.0, gTau = 0.0;
    if (i < n) {
        double* gd = grad + 7 * (size_t)i;
        const double s_ct = gd[0], s_qf = gd[1], s_sL = gd[5], s_sT = gd[6];
        const double* pd = dep + 7 * (size_t)i;
        const double q0 = pd[1], x0 = pd[2], el0 = pd[5], et0 = pd[6];
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
        double gx = 0.0;  // x' = x_response: x enters through the drift time only
        if (found >= 0) {
            const double respx = dd.xr[found][1];
            const double dtm = fabs((respx - x0) / dd.speed);
            const double dtdx = (x0 > respx ? 1.0 : -1.0) / dd.speed;  // d(dt)/dx
            if (dir > 0) {
                // t' = t + dt, q' = q exp(-dt/lifetime), sL^2 = 2 DL dt + el^2, sT^2 = 2 DT dt + et^2
                const double ex = exp(-dtm / dd.lifetime);
                const double qd = q0 * ex;
                const double sL = sqrt(2.0 * dd.DL * dtm + el0 * el0);
                const double sT = sqrt(2.0 * dd.DT * dtm + et0 * et0);
                const double hL = sL > 0.0 ? s_sL / sL : 0.0;
                const double hT = sT > 0.0 ? s_sT / sT : 0.0;
                const double gdt = s_ct - s_qf * qd / dd.lifetime + hL * dd.DL + hT * dd.DT;
                gx = gdt * dtdx;
                gd[1] = s_qf * ex;
                gd[5] = hL * el0;
                gd[6] = hT * et0;
                gDL = hL * dtm;
                gDT = hT * dtm;
                gTau = s_qf * qd * dtm / (dd.lifetime * dd.lifetime);
            }
            else {
                gx = -s_ct * dtdx;  // t' = t - dt in the response region
            }
        }
        gd[2] = gx;
    }
    __shared__ double s_glob[8][3];
    gDL = warp_sum_d(gDL);
    gDT = warp_sum_d(gDT);
    gTau = warp_sum_d(gTau);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        s_glob[w][0] = gDL;
        s_glob[w][1] = gDT;
        s_glob[w][2] = gTau;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += s_glob[k][threadIdx.x];
        if (v != 0.0) atomicAdd(gglob + threadIdx.x, v);
    }
}

void launch_adj_gather(const double* depos, int n, const DriftDev& dd, int do_drift, const PlaneSet& ps,
                       const AdjSet& as, double drift_speed, const PatchRec* rec, const float* dQ, double* grad,
                       double* gglob, cudaStream_t s, const double* qscale)
{
    if (n <= 0) return;
    const int blocks = (n + kGatherWarps - 1) / kGatherWarps;
    k_adj_gather<<<blocks, kGatherWarps * 32, 0, s>>>(n, ps, as, 1.0 / drift_speed, rec, dQ, grad, qscale);
    if (do_drift) k_adj_drift<<<(n + 255) / 256, 256, 0, s>>>(depos, n, dd, grad, gglob);
}

}  // namespace wctb200
