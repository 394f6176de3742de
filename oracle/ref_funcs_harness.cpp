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
// generator's spectrum (GeneratorN::spec, aux/src/NoiseTools.cxx:178-204),
// Drifter::insert with its Xregion helpers (gen/src/Drifter.cxx:22-60,127-196;
// gen/inc/WireCellGen/Drifter.h), BinnedDiffusion_transform::add
// (gen/src/BinnedDiffusion_transform.cxx:37-92) over the reference's IDepo and
// SimpleDepo (iface/inc/WireCellIface/IDepo.h, aux/inc/WireCellAux/SimpleDepo.h,
// aux/src/SimpleDepo.cxx), and Pimpos
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
#include <algorithm>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "WireCellIface/IData.h"
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

// ---- Drifter::insert and BinnedDiffusion_transform::add ----
// The depo interface and its plain implementation are the reference's own
// (iface/inc/WireCellIface/IData.h compiles as it is; IDepo and SimpleDepo
// are cut out of their headers, whose Point.h include needs jsoncpp).
#include "idepo_class.inc"
namespace Aux {
#include "simpledepo_class.inc"
}
// IRandom::binomial (iface/inc/WireCellIface/IRandom.h), the one call of
// Drifter::insert into its random source, when "fluctuate" is on.
class IRandom {
   public:
    typedef std::shared_ptr<IRandom> pointer;
    virtual ~IRandom() {}
    virtual int binomial(int max, double prob) = 0;
};
// The configuration values that Drifter::Xregion's constructor reads
// (Json::Value's operator[], isNull and asDouble).
struct ConfigValue {
    bool null{true};
    double v{0};
    bool isNull() const { return null; }
    double asDouble() const { return v; }
};
struct Configuration {
    std::map<std::string, ConfigValue> m;
    ConfigValue operator[](const char* k) const
    {
        auto it = m.find(k);
        return it == m.end() ? ConfigValue{} : it->second;
    }
};
namespace Gen {
// the members of gen/inc/WireCellGen/Drifter.h that Drifter::insert uses;
// the nested helper types are the header's own text
class Drifter {
   public:
    typedef IDepo::pointer input_pointer;
    bool insert(const input_pointer& depo);
    IRandom::pointer m_rng;
    double m_DL, m_DT;
    double m_lifetime;
    bool m_fluctuate;
    double m_speed;
    double m_toffset;
#include "drifter_structs.inc"
    std::vector<Xregion> m_xregions;
};
// the members of GaussianDiffusion (gen/inc/WireCellGen/GaussianDiffusion.h:80)
// and BinnedDiffusion_transform (gen/inc/WireCellGen/BinnedDiffusion_transform.h:105-121)
// that BinnedDiffusion_transform::add uses
class GaussianDiffusion {
   public:
    GaussianDiffusion(const IDepo::pointer& depo, const GausDesc& time_desc, const GausDesc& pitch_desc)
      : m_deposition(depo), m_time_desc(time_desc), m_pitch_desc(pitch_desc)
    {
    }
    IDepo::pointer m_deposition;
    GausDesc m_time_desc, m_pitch_desc;
};
class BinnedDiffusion_transform {
   public:
    BinnedDiffusion_transform(const Pimpos& pimpos, const Binning& tbins, double nsigma)
      : m_pimpos(pimpos), m_tbins(tbins), m_nsigma(nsigma)
    {
    }
    bool add(IDepo::pointer depo, double sigma_time, double sigma_pitch);
    const Pimpos& m_pimpos;
    const Binning& m_tbins;
    double m_nsigma;
    std::set<std::shared_ptr<GaussianDiffusion> > m_diffs;
    int m_outside_pitch{0};
    int m_outside_time{0};
};
}  // namespace Gen
}  // namespace WireCell
WireCell::IDepo::~IDepo() {}

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
#include "simpledepo_fns.inc"
#include "drifter_fns.inc"
#include "bdt_add.inc"

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

// Drifter::insert (gen/src/Drifter.cxx:127-196) of one depo, fluctuation
// off: xr [nxr][3] (anode, response, cathode) as Xregion configurations,
// depo (t, q, x, y, z, extent_long, extent_tran).  Returns 1 and the drifted
// depo in out (same layout) when insert keeps it, else 0.
int ref_drift_one(const double* xr, int nxr, double DL, double DT, double lifetime, double speed, double toffset,
                  const double* depo, double* out)
{
    Gen::Drifter d;
    d.m_DL = DL;
    d.m_DT = DT;
    d.m_lifetime = lifetime;
    d.m_fluctuate = false;
    d.m_speed = speed;
    d.m_toffset = toffset;
    for (int k = 0; k < nxr; ++k) {
        Configuration c;
        c.m["anode"] = ConfigValue{false, xr[3 * k]};
        c.m["response"] = ConfigValue{false, xr[3 * k + 1]};
        c.m["cathode"] = ConfigValue{false, xr[3 * k + 2]};
        d.m_xregions.emplace_back(c);
    }
    auto in = std::make_shared<Aux::SimpleDepo>(depo[0], Point(depo[2], depo[3], depo[4]), depo[1], nullptr, depo[5],
                                                depo[6], 7);
    if (!d.insert(in)) return 0;
    for (auto& x : d.m_xregions)
        for (auto& o : x.depos) {
            out[0] = o->time();
            out[1] = o->charge();
            out[2] = o->pos().x();
            out[3] = o->pos().y();
            out[4] = o->pos().z();
            out[5] = o->extent_long();
            out[6] = o->extent_tran();
            return 1;
        }
    return -1;
}
// BinnedDiffusion_transform::add (gen/src/BinnedDiffusion_transform.cxx:37-92)
// of one depo on a plane (the Pimpos arguments as ref_pimpos) and the
// readout binning (ntbins over [tmin, tmax]); sigma_time and sigma_pitch as
// DepoTransform passes them.  Returns 1 when added; counters[0..1] get
// m_outside_time and m_outside_pitch.
int ref_bdt_add(int nwires, double minp, double maxp, const double* wire, const double* pitch, const double* origin,
                int nimp, int ntbins, double tmin, double tmax, double nsigma, const double* depo, double sigma_time,
                double sigma_pitch, int* counters)
{
    Pimpos pim(nwires, minp, maxp, Vector(wire[0], wire[1], wire[2]), Vector(pitch[0], pitch[1], pitch[2]),
               Point(origin[0], origin[1], origin[2]), nimp);
    Binning tb(ntbins, tmin, tmax);
    Gen::BinnedDiffusion_transform bd(pim, tb, nsigma);
    auto in = std::make_shared<Aux::SimpleDepo>(depo[0], Point(depo[2], depo[3], depo[4]), depo[1], nullptr, depo[5],
                                                depo[6], 7);
    const bool ok = bd.add(in, sigma_time, sigma_pitch);
    counters[0] = bd.m_outside_time;
    counters[1] = bd.m_outside_pitch;
    return ok ? 1 : 0;
}
}
