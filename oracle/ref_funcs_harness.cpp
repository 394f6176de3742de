// TEST INFRASTRUCTURE ONLY.
// Harness around reference functions that compile on their own: the
// GausDesc struct and its sample/binint/weight
// (gen/inc/WireCellGen/GaussianDiffusion.h:20-63,
// gen/src/GaussianDiffusion.cxx:8-92), Waveform::edge
// (util/src/Waveform.cxx:136-153) and Response::coldelec
// (util/src/Response.cxx:311-340).  oracle/extract_ref.py cuts them out of
// the reference tree into oracle/_ref/*.inc and oracle/Makefile compiles this
// file with them into oracle/_ref/libref_funcs.so.  They pin the oracle's bin
// integrals and impact weights, its trace edges and the noise model's
// cold-electronics response to the reference's compiled code.
#include <cmath>
#include <iostream>
#include <utility>
#include <vector>

#include "WireCellUtil/Units.h"
#include "WireCellUtil/Waveform.h"

namespace WireCell {
namespace Gen {
#include "gausdesc_struct.inc"
}
namespace Response {
double coldelec(double time, double gain, double shaping);
}
}  // namespace WireCell

using namespace WireCell;
using namespace std;

#include "gausdesc_fns.inc"
#include "waveform_edge.inc"
#include "coldelec.inc"

extern "C" {
// Length of the result; out must hold max(nbins, 1) values.
int ref_gd_binint(double center, double sigma, double start, double step, int nbins, double* out)
{
    auto v = Gen::GausDesc(center, sigma).binint(start, step, nbins);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return (int)v.size();
}
int ref_gd_weight(double center, double sigma, double start, double step, int nbins, const double* pvec,
                  double* out)
{
    std::vector<double> p(pvec, pvec + nbins);
    auto v = Gen::GausDesc(center, sigma).weight(start, step, nbins, p);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return (int)v.size();
}
double ref_gd_distance(double center, double sigma, double x) { return Gen::GausDesc(center, sigma).distance(x); }
void ref_gd_sigma_range(double center, double sigma, double nsigma, double* out)
{
    auto r = Gen::GausDesc(center, sigma).sigma_range(nsigma);
    out[0] = r.first;
    out[1] = r.second;
}
void ref_wave_edge(const float* wave, int n, int* out)
{
    Waveform::realseq_t w(wave, wave + n);
    auto r = Waveform::edge(w);
    out[0] = r.first;
    out[1] = r.second;
}
double ref_coldelec(double time, double gain, double shaping) { return Response::coldelec(time, gain, shaping); }
}
