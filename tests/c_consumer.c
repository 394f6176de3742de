/* A plain C99 consumer of the C ABI (include/wctb200.h), linked against
 * libwctb200.so the way a C or C++ host framework links it.  It calls only
 * host-side entry points, so it runs without a GPU:
 *
 *   c_consumer IN OUT
 *
 * IN (native doubles): npaths, nsamples, pitch, tstart, period,
 * overall_short_padding, tick, nticks, nshort_samples, nrel, then pitchpos
 * [npaths], current [npaths][nsamples], one short response [nshort_samples],
 * relative pitches [nrel].
 *
 * OUT (native doubles): status of a call with null arguments, whether it set
 * a message, wct_fft_best_length of 964+20 (keep parity) and 3334, then
 * wct_pir_info (pitch, impact, half extent, nwires, nimp_per_wire, npaths,
 * nticks, waveform_pad), closest() per relative pitch (path index or -1 -
 * status), and every path's waveform [npaths][nticks]. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wctb200.h"

static int read_doubles(FILE* f, double* out, size_t n) { return fread(out, sizeof(double), n, f) == n; }

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* in = fopen(argv[1], "rb");
    if (!in) return 2;
    double hdr[10];
    if (!read_doubles(in, hdr, 10)) return 2;
    const int npaths = (int)hdr[0], nsamples = (int)hdr[1], nticks = (int)hdr[7], nshort = (int)hdr[8];
    const int nrel = (int)hdr[9];
    double* pitchpos = malloc(sizeof(double) * npaths);
    double* current = malloc(sizeof(double) * (size_t)npaths * nsamples);
    double* shortw = malloc(sizeof(double) * (nshort > 0 ? nshort : 1));
    double* rel = malloc(sizeof(double) * (nrel > 0 ? nrel : 1));
    if (!read_doubles(in, pitchpos, npaths) || !read_doubles(in, current, (size_t)npaths * nsamples) ||
        !read_doubles(in, shortw, nshort) || !read_doubles(in, rel, nrel))
        return 2;
    fclose(in);

    FILE* out = fopen(argv[2], "wb");
    if (!out) return 2;
    double v;

    /* errors are status codes with a message, never a crash */
    wct_pir* none = NULL;
    v = wct_pir_create(NULL, 0, NULL, NULL, 1.0, 1.0, 10, &none);
    fwrite(&v, sizeof v, 1, out);
    v = strlen(wct_last_error()) > 0;
    fwrite(&v, sizeof v, 1, out);
    v = (double)wct_fft_best_length(964 + 20, 1);
    fwrite(&v, sizeof v, 1, out);
    v = (double)wct_fft_best_length(3334, 0);
    fwrite(&v, sizeof v, 1, out);

    wct_fr_plane fr;
    fr.npaths = npaths;
    fr.nsamples = nsamples;
    fr.pitchpos = pitchpos;
    fr.current = current;
    fr.pitch = hdr[2];
    fr.tstart = hdr[3];
    fr.period = hdr[4];
    const int slen = nshort;
    wct_pir* pir = NULL;
    if (wct_pir_create(&fr, nshort > 0 ? 1 : 0, &slen, shortw, hdr[5], hdr[6], nticks, &pir) != WCT_OK) return 3;

    double pitch, impact, half;
    int nw, nimp, np, nt, wpad;
    if (wct_pir_info(pir, &pitch, &impact, &half, &nw, &nimp, &np, &nt, &wpad) != WCT_OK) return 4;
    double info[8] = {pitch, impact, half, nw, nimp, np, nt, wpad};
    fwrite(info, sizeof(double), 8, out);
    for (int i = 0; i < nrel; ++i) {
        int path = -1;
        const int rc = wct_pir_closest(pir, rel[i], &path);
        v = rc == WCT_OK ? path : -1 - rc;
        fwrite(&v, sizeof v, 1, out);
    }
    float* wave = malloc(sizeof(float) * nt);
    for (int p = 0; p < np; ++p) {
        if (wct_pir_waveform(pir, p, wave) != WCT_OK) return 5;
        for (int k = 0; k < nt; ++k) {
            v = wave[k];
            fwrite(&v, sizeof v, 1, out);
        }
    }
    wct_pir_destroy(pir);
    fclose(out);
    free(wave);
    free(pitchpos);
    free(current);
    free(shortw);
    free(rel);
    return 0;
}
