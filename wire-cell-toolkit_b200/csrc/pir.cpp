#include "pir.hpp"

#include "fft_lengths.h"

#include <algorithm>

namespace wctb200 {

static const size_t kAny[] = {WCT_FFT_LENGTHS_ANY};
static const size_t kEven[] = {WCT_FFT_LENGTHS_EVEN};
static const size_t kOdd[] = {WCT_FFT_LENGTHS_ODD};

template <size_t N>
static size_t pick(const size_t (&t)[N], size_t n)
{
    if (n <= t[N - 1])
        for (size_t i = 0; i < N; ++i)
            if (t[i] >= n) return t[i];
    return n;
}

size_t fft_best_length(size_t n, bool keep_odd_even)
{
    if (!keep_odd_even) return pick(kAny, n);
    return (n % 2 == 0) ? pick(kEven, n) : pick(kOdd, n);
}

std::pair<int, int> Pir::closest_wire_impact(double relpitch) const
{
    const int center_wire = nwires() / 2;
    const int relwire = int(std::round(relpitch / pitch));
    const int wire_index = center_wire + relwire;
    const double remainder = relpitch - relwire * pitch;
    const int impact_index = int(std::round(remainder / impact)) + nimp_per_wire() / 2;
    return {wire_index, impact_index};
}

int Pir::closest(double relpitch) const
{
    if (relpitch < -half_extent || relpitch > half_extent) return -1;
    auto wi = closest_wire_impact(relpitch);
    if (wi.first < 0 || wi.first >= (int)bywire.size()) return -1;
    const auto& region = bywire[wi.first];
    if (wi.second < 0 || wi.second >= (int)region.size()) return -1;
    const int irind = region[wi.second];
    if (irind < 0 || irind >= (int)waveform.size()) return -1;
    return irind;
}

Pir build_pir_layout(int npaths, int nsamples, const double* pitchpos, double fr_pitch, double tstart,
                     double period, double overall_short_padding, double tick, int nticks)
{
    const int n_per = 6;  // six paths per wire region (PlaneImpactResponse.cxx:164)
    if (npaths < n_per || npaths % n_per) throw std::runtime_error("field response must hold 6 paths per wire");
    if (!(fr_pitch > 0.0) || !(period > 0.0) || !(tick > 0.0))
        throw std::runtime_error("field response pitch, period and tick must be positive");
    Pir p;
    p.nticks = nticks;
    p.tick = tick;
    p.waveform_pad = (int)(overall_short_padding / tick);
    const size_t n_short = fft_best_length((size_t)(overall_short_padding / tick), false);
    p.n_short = (int)n_short;
    const int n_wires = npaths / n_per;
    const int n_wires_half = n_wires / 2;
    p.impact = std::abs(pitchpos[1] - pitchpos[0]);
    p.half_extent = std::max(std::abs(pitchpos[0]), std::abs(pitchpos[npaths - 1]));
    p.pitch = 2.0 * std::abs(pitchpos[n_per - 1] - pitchpos[0]);
    // every sample of the field response must land in the short window (:196-205);
    // sample times grow with the index, so the first and the last decide
    const double rawmax = tstart + nsamples * period;
    const double rawbs = (rawmax - tstart) / nsamples;
    for (int r = 0; r < nsamples; r += std::max(1, nsamples - 1)) {
        const double time = tstart + (r + 0.5) * rawbs;  // Binning::center
        if (!(time >= 0.0)) throw std::runtime_error("out of bounds field response (sample before t = 0)");
        if ((size_t)(time / tick) >= n_short) throw std::runtime_error("out of bounds field response");
    }
    const double oopsilon = 1e-15 * fr_pitch;
    std::map<int, std::vector<int>> wire_to_ind;
    for (int ip = 0; ip < npaths; ++ip)
        wire_to_ind[int(std::ceil((pitchpos[ip] - oopsilon) / fr_pitch))].push_back(ip);
    for (int irel = -n_wires_half; irel <= n_wires_half; ++irel) {
        const auto& direct = wire_to_ind[irel];
        const auto& other = wire_to_ind[-irel];
        std::vector<int> idx(direct.begin(), direct.end());
        if (!other.empty())
            for (auto it = other.rbegin() + 1; it != other.rend(); ++it) idx.push_back(*it);
        p.bywire.push_back(idx);
    }
    p.waveform.assign(npaths, std::vector<float>(nticks, 0.0f));
    return p;
}

Pir build_pir(int npaths, int nsamples, const double* pitchpos, const double* current, double fr_pitch,
              double tstart, double period, const std::vector<std::vector<double>>& shorts,
              double overall_short_padding, double tick, int nticks)
{
    Pir p = build_pir_layout(npaths, nsamples, pitchpos, fr_pitch, tstart, period, overall_short_padding, tick,
                             nticks);
    const size_t n_short = (size_t)p.n_short;
    // circular product of the short responses, each cut or zero padded to n_short
    std::vector<double> kern(n_short, 0.0);
    kern[0] = 1.0;
    for (const auto& sw : shorts) {
        std::vector<double> s(n_short, 0.0);
        for (size_t i = 0; i < std::min(n_short, sw.size()); ++i) s[i] = sw[i];
        std::vector<double> out(n_short, 0.0);
        for (size_t a = 0; a < n_short; ++a) {
            if (kern[a] == 0.0) continue;
            for (size_t b = 0; b < n_short; ++b) out[(a + b) % n_short] += kern[a] * s[b];
        }
        kern.swap(out);
    }
    const double rawmax = tstart + nsamples * period;
    const double rawbs = (rawmax - tstart) / nsamples;
    for (int ip = 0; ip < npaths; ++ip) {
        std::vector<double> wave(n_short, 0.0);
        for (int r = 0; r < nsamples; ++r) {
            const double time = tstart + (r + 0.5) * rawbs;  // Binning::center
            if (!(time >= 0.0)) throw std::runtime_error("out of bounds field response (sample before t = 0)");
            const size_t bin = time / tick;
            if (bin >= n_short) throw std::runtime_error("out of bounds field response");
            wave[bin] += current[(size_t)ip * nsamples + r] * period;
        }
        std::vector<double> wf(n_short, 0.0);
        if (shorts.empty()) wf = wave;
        else
            for (size_t a = 0; a < n_short; ++a) {
                if (wave[a] == 0.0) continue;
                for (size_t b = 0; b < n_short; ++b) wf[(a + b) % n_short] += wave[a] * kern[b];
            }
        for (int k = 0; k < nticks && k < (int)n_short; ++k) p.waveform[ip][k] = (float)wf[k];
    }
    return p;
}

void set_long_responses(Pir& p, const std::vector<std::vector<double>>& longs, double long_padding)
{
    p.long_wf.clear();
    p.long_pad = 0;
    if (longs.empty()) return;
    const size_t n = fft_best_length((size_t)p.nticks, false);
    std::vector<double> acc(n, 0.0);
    acc[0] = 1.0;
    for (const auto& lw : longs) {
        std::vector<double> w(n, 0.0);
        for (size_t i = 0; i < std::min(n, lw.size()); ++i) w[i] = lw[i];
        std::vector<double> out(n, 0.0);
        for (size_t a = 0; a < n; ++a) {
            if (acc[a] == 0.0) continue;
            for (size_t b = 0; b < n; ++b) {
                if (w[b] == 0.0) continue;
                out[(a + b) % n] += acc[a] * w[b];
            }
        }
        acc.swap(out);
    }
    p.long_wf.assign(acc.begin(), acc.end());
    p.long_pad = (int)(long_padding / p.tick);
}

}  // namespace wctb200
