// Device data structures and launcher declarations for the DepoTransform
// forward path.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fft.cuh"

namespace wctb200 {

// Drifter configuration (gen/src/Drifter.cxx:62-123).
struct DriftDev {
    double DL, DT, lifetime, speed, toffset;
    int nxr;
    double xr[8][3];  // anode, response, cathode
};

// One wire plane as seen by the rasteriser: pitch axis / origin of its
// Pimpos (util/src/Pimpos.cxx:5-33), its impact binning and the face's
// sensitive box (gen/src/AnodePlane.cxx:259-290).
struct PlaneDev {
    double ax, ay, az;        // unit pitch axis
    double ox, oy, oz;        // Pimpos origin
    int nwires, nimp;
    int imp_nbins;
    double imp_min, imp_max, imp_bs;
    int have_bb;
    double bb_lo[3], bb_hi[3];
    int depo_slot;            // which drifted-depo flag array applies (face)
};

// Readout time binning (gen/src/DepoTransform.cxx:180).
struct TimeDev {
    int nbins;
    double tmin, tmax, bs;
};

// Per (plane, depo) patch description, written by the prep kernel.
// np == 0 marks a depo that does not contribute to the plane.
struct PatchRec {
    int toff, poff;
    unsigned short nt, np;
    float tcr;   // center_time - edge(toff)
    float pcr;   // center_pitch - edge(poff)
    float st;    // sigma_time
    float sp;    // sigma_pitch
    float q;     // charge
};
static_assert(sizeof(PatchRec) == 32, "PatchRec layout");

// Per-plane window reduction (BinnedDiffusion_transform.cxx:416-464).
struct WindowDev {
    unsigned long long pmin, pmax, tmin, tmax;  // order-preserving double keys
    int nadded, out_time, out_pitch, oversize;
};

constexpr int kMaxPatchT = 512;   // raster limit on ticks per patch
constexpr int kMaxPatchP = 256;   // raster limit on impact bins per patch

// ---- launchers (kernels.cu) ----
void launch_drift(const double* depos, int n, const DriftDev& dd, int do_drift, double* out, unsigned char* valid,
                  cudaStream_t s);
void launch_prep(const double* depos, const unsigned char* valid, int n, const PlaneDev& pl, const TimeDev& tb,
                 double drift_speed, double nsigma, PatchRec* rec, WindowDev* win, cudaStream_t s);
void launch_raster(const PatchRec* rec, int n, const PlaneDev& pl, const TimeDev& tb, int ngroups, int row0,
                   int nrows, int col0, int ldq, float* Q, WindowDev* win, cudaStream_t s);
void launch_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows,
                      const FftDesc& d, cudaStream_t s);
void launch_wire_conv(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                      int nrows_out, int M, cudaStream_t s);
void launch_irfft_rows(const float2* Vh, int nrows, const FftDesc& d, int wire0, int wlo, int whi, int tick0,
                       int ncols, int nticks, float* frame, cudaStream_t s);

}  // namespace wctb200
