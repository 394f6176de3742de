// Host-side code of the library under AddressSanitizer and
// UndefinedBehaviorSanitizer (built and run by tests/test_host_sanitize.py):
// the JSON configuration reader (csrc/json.hpp) on valid, invalid, deeply
// nested and randomly mutated documents, and the PlaneImpactResponse build,
// closest() lookup and long-response product (csrc/pir.cpp) over a range of
// field-response geometries.  Exit status 0 and "ok" on success; a sanitizer
// report aborts the process.
#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "json.hpp"
#include "pir.hpp"

using namespace wctb200;

static int failures = 0;
#define CHECK(c)                                                              \
    do {                                                                      \
        if (!(c)) {                                                           \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #c); \
            ++failures;                                                       \
        }                                                                     \
    } while (0)

static bool parses(const std::string& s)
{
    try {
        json::parse(s);
        return true;
    }
    catch (const std::runtime_error&) {
        return false;
    }
}

static void json_cases()
{
    const std::string cfg =
        "{\"nsigma\": 3.0, \"fluctuate\": false, \"start_time\": -1.5e-3, \"readout_time\": 5000000.0, "
        "\"tick\": 500, \"drift_speed\": 0.0016, \"first_frame_number\": 0, \"anode\": \"AnodePlane:a\", "
        "\"pirs\": [\"PlaneImpactResponse:u\", \"PlaneImpactResponse:v\", \"PlaneImpactResponse:w\"], "
        "\"drifter\": {\"DL\": 7.2e-9, \"DT\": 1.2e-8, \"lifetime\": 1e7, \"xregions\": [{\"anode\": 0, "
        "\"response\": 100.0, \"cathode\": 2500.0}]}, \"name\": \"a\\\"b\\u00e9\\n\", \"seed\": null}";
    json::Value v = json::parse(cfg);
    CHECK(v["nsigma"].as_number(0) == 3.0);
    CHECK(v["start_time"].as_number(0) == -1.5e-3);
    CHECK(v["tick"].as_number(0) == 500.0);
    CHECK(v["drift_speed"].as_number(0) == 0.0016);
    CHECK(v["pirs"].arr.size() == 3);
    CHECK(v["drifter"]["xregions"].arr[0]["cathode"].as_number(0) == 2500.0);
    CHECK(v["name"].as_string("") == std::string("a\"b\xc3\xa9\n"));
    CHECK(v["seed"].is_null());
    CHECK(v["missing"].as_number(7.0) == 7.0);

    for (const char* good : {"0", "-0", "1e5", "1E+5", "2.5e-3", "[]", "{}", "[[], {}]", " \t\n[1, 2] ", "\"\""})
        CHECK(parses(good));
    for (const char* bad : {"", "{", "}", "[1,]", "[1 2]", "01", "[01]", "1.", ".5", "-", "+1", "1e", "1e+",
                            "nan", "NaN", "Infinity", "-Infinity", "0x10", "1e999", "{\"a\" 1}", "{1: 2}",
                            "\"abc", "\"\\", "tru", "[true false]", "{\"a\": 1,}"})
        CHECK(!parses(bad));

    // nesting: at the limit it parses, beyond it is an error (not a stack overflow)
    const int lim = json::Parser::kMaxDepth;
    CHECK(parses(std::string(lim, '[') + std::string(lim, ']')));
    CHECK(!parses(std::string(lim + 1, '[') + std::string(lim + 1, ']')));
    CHECK(!parses(std::string(1000000, '[')));
    CHECK(!parses(std::string(500000, '{')));

    // random mutations of the configuration: parse or throw, nothing else
    std::mt19937 rng(12345);
    const std::string alphabet = "{}[]\",:.-+eE0123456789 \\tfnu\x01\xff";
    int ok = 0;
    for (int it = 0; it < 20000; ++it) {
        std::string s = cfg;
        const int nmut = 1 + rng() % 4;
        for (int m = 0; m < nmut && !s.empty(); ++m) {
            const size_t at = rng() % s.size();
            switch (rng() % 4) {
                case 0: s[at] = alphabet[rng() % alphabet.size()]; break;
                case 1: s.insert(s.begin() + at, alphabet[rng() % alphabet.size()]); break;
                case 2: s.erase(at, 1 + rng() % 8); break;
                default: s.resize(at); break;
            }
        }
        ok += parses(s);
    }
    CHECK(ok > 0 && ok < 20000);
}

static void pir_cases()
{
    std::mt19937 rng(777);
    for (int nwire_half : {0, 1, 2, 5, 10}) {
        for (int nsamples : {50, 400, 1000}) {
            const double pitch = 3.0 + (rng() % 300) * 0.01;
            const double period = 100.0;
            std::vector<double> pp, cur;
            for (int k = -nwire_half; k <= nwire_half; ++k)
                for (int m = 0; m < 6; ++m) pp.push_back((k - 0.5 + m / 10.0) * pitch - 1e-9 * pitch);
            const int npaths = (int)pp.size();
            for (int p = 0; p < npaths; ++p)
                for (int r = 0; r < nsamples; ++r) {
                    const double u = ((r + 0.5) * period - 0.4 * nsamples * period) / (0.05 * nsamples * period);
                    cur.push_back(std::exp(-0.5 * u * u) * std::exp(-std::fabs(pp[p] / pitch) / 2));
                }
            std::vector<std::vector<double>> shorts;
            if (nsamples != 50) {
                std::vector<double> sh(180 + rng() % 60);
                for (size_t i = 0; i < sh.size(); ++i) sh[i] = std::exp(-0.05 * i) * (double)i;
                shorts.push_back(sh);
            }
            for (int nticks : {100, 1000, 3000}) {
                Pir p = build_pir(npaths, nsamples, pp.data(), cur.data(), pitch, 0.0, period, shorts, 100e3, 500.0,
                                  nticks);
                CHECK(p.nwires() == 2 * nwire_half + 1);
                CHECK((int)p.waveform.size() == npaths);
                for (int i = 0; i < 2000; ++i) {
                    const double rel = (2.0 * (rng() / (double)rng.max()) - 1.0) * 1.2 * p.half_extent;
                    const int k = p.closest(rel);
                    CHECK(k >= -1 && k < npaths);
                    if (std::fabs(rel) > p.half_extent) CHECK(k == -1);
                }
                if (nticks > 1000) continue;  // the direct long-response product is O(n^2)
                std::vector<std::vector<double>> longs;
                for (int L : {1, 37, 5000}) {
                    std::vector<double> w(L);
                    for (int i = 0; i < L; ++i) w[i] = std::exp(-0.01 * i);
                    longs.push_back(w);
                }
                set_long_responses(p, longs, 1.5e6);
                CHECK(p.long_wf.size() == fft_best_length((size_t)nticks, false));
                set_long_responses(p, {}, 0.0);
                CHECK(p.long_wf.empty());
            }
        }
    }
    // inconsistent responses are exceptions
    std::vector<double> pp(5, 0.0), cur(5 * 10, 0.0);
    bool threw = false;
    try {
        build_pir(5, 10, pp.data(), cur.data(), 3.0, 0.0, 100.0, {}, 100e3, 500.0, 100);
    }
    catch (const std::runtime_error&) {
        threw = true;
    }
    CHECK(threw);
}

int main()
{
    json_cases();
    pir_cases();
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
