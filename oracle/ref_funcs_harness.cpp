// TEST INFRASTRUCTURE ONLY.
// Harness around reference functions that compile on their own: the
// GausDesc struct and its sample/binint/weight
// (gen/inc/WireCellGen/GaussianDiffusion.h:20-63,
// gen/src/GaussianDiffusion.cxx:8-92), Waveform::edge
// (util/src/Waveform.cxx:136-153), Response::coldelec
// (util/src/Response.cxx:311-340), Digitizer::digitize
// (gen/src/Digitizer.cxx:77-93), EmpiricalNoiseModel's frequency grid,
// spectrum resampling and wire-length interpolation
// (gen/src/EmpiricalNoiseModel.cxx:55-147,232-275), the group
// spectra of GroupNoiseModel (gen/src/GroupNoiseModel.cxx:97-146 on
// util/inc/WireCellUtil/Interpolate.h and Spectrum.h), the noise
// generator's spectrum (GeneratorN::spec, aux/src/NoiseTools.cxx:178-204) and
// Pimpos
// (util/inc/WireCellUtil/Pimpos.h,
// util/src/Pimpos.cxx:5-68).  oracle/extract_ref.py cuts them out of the
// reference tree into oracle/_ref/*.inc and oracle/Makefile compiles this
// file with them into oracle/_ref/libref_funcs.so.  They pin the oracle's bin
// integrals and impact weights, its trace edges, its plane geometry (pitch
// coordinate, wire and impact binning), its ADC arithmetic and the noise
// model's resampling and cold-electronics response to the reference's
// compiled code.  Point and
// Vector are the reference's D3Vector<double> (util/inc/WireCellUtil/Point.h
// names them so; that header itself needs jsoncpp).
#include <cmath>
#include <complex>
#include <functional>
#include <iostream>
#include <map>
#include <stdexcept>
#include <unordered_map>
#include <utility>
#include <vector>

#include "WireCellUtil/Binning.h"
#include "WireCellUtil/Interpolate.h"
#include "WireCellUtil/D3Vector.h"
#include "WireCellUtil/Units.h"
#include "WireCellUtil/Waveform.h"

namespace WireCell {
typedef D3Vector<double> Point;
typedef Point Vector;
#include "pimpos_class.inc"
namespace Gen {
#include "gausdesc_struct.inc"
// the members that Digitizer::digitize reads (gen/inc/WireCellGen/Digitizer.h:43-56)
struct Digitizer {
    int m_resolution{12};
    std::vector<double> m_fullscale;
    bool m_round{false};
    double digitize(double voltage);
};
// the members that EmpiricalNoiseModel::gen_elec_resp_default and resample
// use (gen/inc/WireCellGen/EmpiricalNoiseModel.h:65-125; amplitude_t is
// IChannelSpectrum's)
class EmpiricalNoiseModel {
   public:
    typedef std::vector<float> amplitude_t;
#include "noise_spectrum.inc"
    void gen_elec_resp_default();
    void resample(NoiseSpectrum& spectrum) const;
    using spectrum_data_t = std::pair<double, amplitude_t>;
    spectrum_data_t interpolate_wire_length(int plane, double wire_length) const;
    int m_fft_length{0};
    double m_period{0};
    Waveform::realseq_t m_elec_resp_freq;
    std::map<int, std::vector<NoiseSpectrum*> > m_spectral_data;
};
}
namespace Response {
double coldelec(double time, double gain, double shaping);
}
// Spectrum's extrap and alias raise their errors with the toolkit's THROW
// (WireCellUtil/Exceptions.h, which needs Boost): a plain exception here.
struct errmsg {
    const char* what;
};
struct ValueError {
    ValueError& operator<<(const errmsg&) { return *this; }
};
#define THROW(e) throw std::runtime_error("reference THROW")
namespace Spectrum {
#include "spectrum_fns.inc"
}
// the parts of aux/inc/WireCellAux/NoiseTools.h:19-20,237-253 that
// GeneratorN::spec uses: its types and the source of normal variates
namespace Aux::NoiseTools {
using real_vector_t = std::vector<float>;
using complex_vector_t = std::vector<std::complex<float> >;
class GeneratorN {
   public:
    using normal_f = std::function<real_vector_t(size_t n)>;
    normal_f normal;
    complex_vector_t spec(const real_vector_t& sigmas);
};
}  // namespace Aux::NoiseTools
}  // namespace WireCell

using namespace WireCell;
using namespace std;

#include "gausdesc_fns.inc"
#include "waveform_edge.inc"
#include "coldelec.inc"
#include "pimpos_fns.inc"
#include "digitize.inc"
#include "noise_fns.inc"
using namespace WireCell::Spectrum;
using namespace WireCell::Aux::NoiseTools;
#include "generatorn.inc"

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
// Digitizer::operator() per sample (gen/src/Digitizer.cxx:126-131): the
// voltage gain * value + baseline (the baseline read into a float), its ADC
// value from digitize(), stored as a float.
void ref_digitize(const float* frame, int nrows, int ncols, const float* row_baseline, double gain, double fs_lo,
                  double fs_hi, int resolution, int round_adc, float* adc)
{
    Gen::Digitizer d;
    d.m_resolution = resolution;
    d.m_fullscale = {fs_lo, fs_hi};
    d.m_round = round_adc != 0;
    for (int r = 0; r < nrows; ++r) {
        const float baseline = row_baseline[r];
        for (int c = 0; c < ncols; ++c) {
            const double voltage = gain * frame[(size_t)r * ncols + c] + baseline;
            adc[(size_t)r * ncols + c] = d.digitize(voltage);
        }
    }
}
// One spectrum of the noise model's "spectra_file" resampled as configure()
// does (gen/src/EmpiricalNoiseModel.cxx:175-188,193-221): the model grid of
// fft_length bins at period; the entry's float fields as read by asFloat.
// Returns the resampled amplitude count (amps_out holds max(fft_length,
// namps)); *constant receives the scaled constant.
int ref_noise_resample(int fft_length, double period, int nsamples, float entry_period, double* constant,
                       const float* freqs, int nfreqs, const float* amps, int namps, float* amps_out)
{
    Gen::EmpiricalNoiseModel m;
    m.m_fft_length = fft_length;
    m.m_period = period;
    m.gen_elec_resp_default();
    Gen::EmpiricalNoiseModel::NoiseSpectrum ns{};
    ns.nsamples = nsamples;
    ns.period = entry_period;
    ns.constant = *constant;
    ns.freqs.assign(freqs, freqs + nfreqs);
    ns.amps.assign(amps, amps + namps);
    m.resample(ns);
    *constant = ns.constant;
    for (size_t i = 0; i < ns.amps.size(); ++i) amps_out[i] = ns.amps[i];
    return (int)ns.amps.size();
}
// EmpiricalNoiseModel::interpolate_wire_length (:232-275) over nspec spectra
// of one plane (in file order: wire lengths ascending), each namps floats.
// Returns 0, or -1 where the reference throws.
int ref_noise_interp(int nspec, const double* wirelen, const double* constant, const float* amps, int namps,
                     double wire_length, double* const_out, float* amps_out)
{
    std::vector<Gen::EmpiricalNoiseModel::NoiseSpectrum> specs(nspec);
    Gen::EmpiricalNoiseModel m;
    for (int k = 0; k < nspec; ++k) {
        specs[k].wirelen = wirelen[k];
        specs[k].constant = constant[k];
        specs[k].amps.assign(amps + (size_t)k * namps, amps + (size_t)(k + 1) * namps);
        m.m_spectral_data[0].push_back(&specs[k]);
    }
    try {
        auto r = m.interpolate_wire_length(0, wire_length);
        *const_out = r.first;
        for (size_t i = 0; i < r.second.size(); ++i) amps_out[i] = r.second[i];
        return 0;
    }
    catch (const std::exception&) {
        return -1;
    }
}
// GeneratorN::spec (aux/src/NoiseTools.cxx:178-204) of n sigmas with the
// given normals (2 (n/2 + (n even)) + 1 of them): the complex spectrum as n
// (re, im) float pairs.  Returns 0, or -1 where the reference throws.
int ref_generator_spec(int n, const float* sigmas, const float* normals, int nnormals, float* out)
{
    Aux::NoiseTools::GeneratorN g;
    g.normal = [&](size_t k) {
        if ((int)k > nnormals) throw std::runtime_error("too few normals");
        return Aux::NoiseTools::real_vector_t(normals, normals + k);
    };
    try {
        auto spec = g.spec(Aux::NoiseTools::real_vector_t(sigmas, sigmas + n));
        for (int i = 0; i < n; ++i) {
            out[2 * i] = spec[i].real();
            out[2 * i + 1] = spec[i].imag();
        }
        return 0;
    }
    catch (const std::exception&) {
        return -1;
    }
}
// The model's frequency grid (gen_elec_resp_default, :55-70), fft_length floats.
void ref_noise_freqs(int fft_length, double period, float* out)
{
    Gen::EmpiricalNoiseModel m;
    m.m_fft_length = fft_length;
    m.m_period = period;
    m.gen_elec_resp_default();
    for (int i = 0; i < fft_length; ++i) out[i] = m.m_elec_resp_freq[i];
}
// GroupNoiseModel::configure's treatment of one spectrum
// (gen/src/GroupNoiseModel.cxx:97-146), restated line for line around the
// reference's irrterp, Spectrum::hermitian_mirror and Spectrum::resample:
// the half spectrum up to Nyquist interpolated onto norig Rayleigh steps,
// mirrored, and resampled to nsamples at tick.  Returns 0, or -1 where the
// reference throws (no points below Nyquist).
int ref_group_spectrum(int norig, double porig, int npts, const float* freqs, const float* amps, double spec_scale,
                       int nsamples, double tick, float* out)
{
    const double Fnyquist = 1.0 / (2 * porig);
    const double Frayleigh = 1.0 / ((size_t)norig * porig);
    std::unordered_map<float, float> pts;
    for (int ind = 0; ind < npts; ++ind) {
        const float freq = freqs[ind];
        if (freq > Fnyquist) continue;
        pts[freq] = spec_scale * amps[ind];
    }
    if (pts.empty()) return -1;
    irrterp<float> terp(pts.begin(), pts.end());
    std::vector<float> sorig(norig, 0);
    terp(sorig.begin(), norig, 0, Frayleigh);
    Spectrum::hermitian_mirror(sorig.begin(), sorig.end());
    std::vector<float> spec(nsamples, 0);
    try {
        Spectrum::resample(sorig.begin(), sorig.end(), spec.begin(), spec.end(), tick / porig);
    }
    catch (const std::exception&) {
        return -1;
    }
    for (int i = 0; i < nsamples; ++i) out[i] = spec[i];
    return 0;
}
// Pimpos of a plane: out = {region nbins, min, max, impact nbins, min, max,
// axis0[3], axis1[3], axis2[3]}; pts [n][3] -> dist [n], the pitch
// coordinate Pimpos::distance(pt, 2).
void ref_pimpos(int nwires, double minp, double maxp, const double* wire, const double* pitch, const double* origin,
                int nbins, int n, const double* pts, double* out, double* dist)
{
    Pimpos p(nwires, minp, maxp, Vector(wire[0], wire[1], wire[2]), Vector(pitch[0], pitch[1], pitch[2]),
             Point(origin[0], origin[1], origin[2]), nbins);
    const Binning& r = p.region_binning();
    const Binning& i = p.impact_binning();
    const double head[6] = {(double)r.nbins(), r.min(), r.max(), (double)i.nbins(), i.min(), i.max()};
    for (int k = 0; k < 6; ++k) out[k] = head[k];
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 3; ++k) out[6 + 3 * a + k] = p.axis(a)[k];
    for (int j = 0; j < n; ++j) dist[j] = p.distance(Point(pts[3 * j], pts[3 * j + 1], pts[3 * j + 2]));
}
}
