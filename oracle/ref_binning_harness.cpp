// TEST INFRASTRUCTURE ONLY.
// Harness around the reference's own header-only Binning
// (util/inc/WireCellUtil/Binning.h), compiled straight from the reference
// source tree by oracle/Makefile into oracle/_ref/. It pins the oracle's and
// the GPU path's bin-index arithmetic (bin, edge, sample_bin_range) and the
// Gaussian helpers (gcumulative, gbounds) to the reference's compiled code.
#include "WireCellUtil/Binning.h"

extern "C" {
int ref_bin(int nbins, double lo, double hi, double v) { return WireCell::Binning(nbins, lo, hi).bin(v); }
double ref_edge(int nbins, double lo, double hi, int i) { return WireCell::Binning(nbins, lo, hi).edge(i); }
double ref_center(int nbins, double lo, double hi, int i) { return WireCell::Binning(nbins, lo, hi).center(i); }
double ref_binsize(int nbins, double lo, double hi) { return WireCell::Binning(nbins, lo, hi).binsize(); }
void ref_sample_bin_range(int nbins, double lo, double hi, double a, double b, int* out)
{
    auto r = WireCell::Binning(nbins, lo, hi).sample_bin_range(a, b);
    out[0] = r.first;
    out[1] = r.second;
}
double ref_gcumulative(double L, double mean, double sigma) { return WireCell::gcumulative(L, mean, sigma); }
double ref_gbounds(double a, double b, double mean, double sigma) { return WireCell::gbounds(a, b, mean, sigma); }
double ref_gaussian_sum(int nbins, double lo, double hi, double mean, double sigma, double* out)
{
    return WireCell::gaussian(out, WireCell::Binning(nbins, lo, hi), mean, sigma);
}
}
