// Host-side PlaneImpactResponse and fft_best_length.
#pragma once

#include <cmath>
#include <cstddef>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace wctb200 {

// util/src/FFTBestLength.cxx:12-59: smallest "fast" FFT size >= n from the
// reference's fixed tables (optionally keeping n's parity).  The window
// indices of ImpactTransform depend on it, so the tables are the same.
size_t fft_best_length(size_t n, bool keep_odd_even);

// PlaneImpactResponse (gen/src/PlaneImpactResponse.cxx:89-320).
struct Pir {
    std::vector<std::vector<float>> waveform;  // [npaths][nticks]  IImpactResponse::waveform()
    std::vector<std::vector<int>> bywire;      // symmetrised wire-region -> path indices
    double pitch{0}, impact{0}, half_extent{0};
    int nticks{0};
    int waveform_pad{0};
    int n_short{0};
    double tick{0};
    // long-range response (IImpactResponse::long_aux_waveform and
    // long_aux_waveform_pad, PlaneImpactResponse.cxx:121-150,252); empty: none
    std::vector<float> long_wf;
    int long_pad{0};

    int nwires() const { return (int)bywire.size(); }
    int nimp_per_wire() const { return bywire.empty() ? 0 : (int)bywire[0].size(); }
    // PlaneImpactResponse::closest_wire_impact, :278-292
    std::pair<int, int> closest_wire_impact(double relpitch) const;
    // PlaneImpactResponse::closest, :294-320; -1 where the reference throws.
    int closest(double relpitch) const;
};

// Everything of PlaneImpactResponse::build_responses but the waveforms
// (left zero): pitch, impact, half extent, the wire grouping of the paths by
// ceil() and its mirror symmetry (:155-268), the short window length, and the
// check that every field-response sample lands in it.
Pir build_pir_layout(int npaths, int nsamples, const double* pitchpos, double fr_pitch, double tstart,
                     double period, double overall_short_padding, double tick, int nticks);

// PlaneImpactResponse::build_responses without long responses.  The
// per-path response is the circular convolution (length n_short) of the
// tick-binned field-response charge with the product of the short responses,
// computed directly in double precision; the reference computes the same
// circular convolution with single-precision DFTs.
Pir build_pir(int npaths, int nsamples, const double* pitchpos, const double* current, double fr_pitch,
              double tstart, double period, const std::vector<std::vector<double>>& shorts,
              double overall_short_padding, double tick, int nticks);

// The long-range response of PlaneImpactResponse::build_responses
// (:121-150): the circular convolution, at length fft_best_length(nticks),
// of the long responses (each cut or zero padded to that length; the
// reference multiplies their single-precision spectra), computed directly in
// double precision; long_pad = long_padding / tick.  No responses: none.
void set_long_responses(Pir& p, const std::vector<std::vector<double>>& longs, double long_padding);

}  // namespace wctb200
