"""TEST INFRASTRUCTURE ONLY.

Cuts self-contained pieces out of the reference source tree, as they are,
into oracle/_ref/ (git-ignored build output) so that oracle/Makefile can
compile them with ref_funcs_harness.cpp.  The surrounding reference files
cannot be compiled here (they include Boost, Eigen, jsoncpp or spdlog
headers); the pieces themselves need only the standard library and the
reference's own header-only Units.h, Waveform.h, Binning.h, D3Vector.h and
Interpolate.h.

  gausdesc_struct.inc  struct GausDesc       gen/inc/WireCellGen/GaussianDiffusion.h
  gausdesc_fns.inc     GausDesc::sample, binint, weight
                                             gen/src/GaussianDiffusion.cxx
  waveform_edge.inc    Waveform::edge        util/src/Waveform.cxx
  coldelec.inc         Response::coldelec    util/src/Response.cxx
  digitize.inc         Digitizer::digitize   gen/src/Digitizer.cxx
  noise_spectrum.inc   struct NoiseSpectrum  gen/inc/WireCellGen/EmpiricalNoiseModel.h
  noise_fns.inc        EmpiricalNoiseModel::gen_elec_resp_default, resample,
                       interpolate_wire_length
                                             gen/src/EmpiricalNoiseModel.cxx
  spectrum_fns.inc     Spectrum::conjugate, hermitian_mirror, interp, extrap,
                       alias, resample       util/inc/WireCellUtil/Spectrum.h
  generatorn.inc       GeneratorN::spec      aux/src/NoiseTools.cxx
  pimpos_class.inc     class Pimpos          util/inc/WireCellUtil/Pimpos.h
  pimpos_fns.inc       Pimpos methods        util/src/Pimpos.cxx (all but its #include)
  idepo_class.inc      class IDepo           iface/inc/WireCellIface/IDepo.h
  simpledepo_class.inc class SimpleDepo      aux/inc/WireCellAux/SimpleDepo.h
  simpledepo_fns.inc   SimpleDepo methods    aux/src/SimpleDepo.cxx (all but its #include)
  drifter_structs.inc  Drifter's DepoTimeCompare, Xregion, IsInsideBulk,
                       IsInsideResp          gen/inc/WireCellGen/Drifter.h
  drifter_fns.inc      DepoTimeCompare::operator(), the Xregion constructor,
                       inside_response, inside_bulk, Drifter::insert
                                             gen/src/Drifter.cxx
  bdt_add.inc          BinnedDiffusion_transform::add
                                             gen/src/BinnedDiffusion_transform.cxx

Each piece is found by its declaration (not by line number) and ends at the
brace that closes it, or at the end of the file for "rest" pieces.

Usage: python extract_ref.py REFERENCE_TREE OUT_DIR"""

import os
import re
import sys

PIECES = {
    "gausdesc_struct.inc": [("gen/inc/WireCellGen/GaussianDiffusion.h", r"^\s*struct GausDesc\s*\{")],
    "gausdesc_fns.inc": [
        ("gen/src/GaussianDiffusion.cxx", r"^std::vector<double> Gen::GausDesc::sample\("),
        ("gen/src/GaussianDiffusion.cxx", r"^std::vector<double> Gen::GausDesc::binint\("),
        ("gen/src/GaussianDiffusion.cxx", r"^std::vector<double> Gen::GausDesc::weight\("),
    ],
    "waveform_edge.inc": [("util/src/Waveform.cxx", r"^std::pair<int, int> WireCell::Waveform::edge\(")],
    "coldelec.inc": [("util/src/Response.cxx", r"^double Response::coldelec\(")],
    "digitize.inc": [("gen/src/Digitizer.cxx", r"^double Gen::Digitizer::digitize\(")],
    "noise_spectrum.inc": [("gen/inc/WireCellGen/EmpiricalNoiseModel.h", r"^\s*struct NoiseSpectrum\s*\{")],
    "noise_fns.inc": [
        ("gen/src/EmpiricalNoiseModel.cxx", r"^void Gen::EmpiricalNoiseModel::gen_elec_resp_default\("),
        ("gen/src/EmpiricalNoiseModel.cxx", r"^void Gen::EmpiricalNoiseModel::resample\("),
        ("gen/src/EmpiricalNoiseModel.cxx",
         r"^Gen::EmpiricalNoiseModel::spectrum_data_t\s*\nGen::EmpiricalNoiseModel::interpolate_wire_length\("),
    ],
    "spectrum_fns.inc": [
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename T>\s*\n\s*std::complex<T> conjugate\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename T> T conjugate\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename It>\s*\n\s*void hermitian_mirror\(It beg"),
        ("util/inc/WireCellUtil/Spectrum.h",
         r"^\s*template<typename InputIt, typename OutputIt>\s*\n\s*OutputIt hermitian_mirror\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename InputIt, typename OutputIt>\s*\n\s*void interp\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename InputIt, typename OutputIt>\s*\n\s*void extrap\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename InputIt, typename OutputIt>\s*\n\s*void alias\("),
        ("util/inc/WireCellUtil/Spectrum.h", r"^\s*template<typename InputIt, typename OutputIt>\s*\n\s*void resample\("),
    ],
    "generatorn.inc": [("aux/src/NoiseTools.cxx", r"^complex_vector_t\s*\nGeneratorN::spec\(")],
    "pimpos_class.inc": [("util/inc/WireCellUtil/Pimpos.h", r"^\s*class Pimpos\s*\{")],
    # the whole file after its one #include line
    "pimpos_fns.inc": [("util/src/Pimpos.cxx", r"^using namespace WireCell;", "rest")],
    "idepo_class.inc": [("iface/inc/WireCellIface/IDepo.h", r"^\s*class IDepo : public IData<IDepo>\s*\{")],
    "simpledepo_class.inc": [("aux/inc/WireCellAux/SimpleDepo.h", r"^\s*class SimpleDepo : public WireCell::IDepo\s*\{")],
    "simpledepo_fns.inc": [("aux/src/SimpleDepo.cxx", r"^using namespace WireCell::Aux;", "rest")],
    "drifter_structs.inc": [
        ("gen/inc/WireCellGen/Drifter.h", r"^\s*struct DepoTimeCompare\s*\{"),
        ("gen/inc/WireCellGen/Drifter.h", r"^\s*struct Xregion\s*\{"),
        ("gen/inc/WireCellGen/Drifter.h", r"^\s*struct IsInsideBulk\s*\{"),
        ("gen/inc/WireCellGen/Drifter.h", r"^\s*struct IsInsideResp\s*\{"),
    ],
    "drifter_fns.inc": [
        ("gen/src/Drifter.cxx", r"^bool Gen::Drifter::DepoTimeCompare::operator\(\)"),
        ("gen/src/Drifter.cxx", r"^Gen::Drifter::Xregion::Xregion\(Configuration cfg\)"),
        ("gen/src/Drifter.cxx", r"^bool Gen::Drifter::Xregion::inside_response\("),
        ("gen/src/Drifter.cxx", r"^bool Gen::Drifter::Xregion::inside_bulk\("),
        ("gen/src/Drifter.cxx", r"^bool Gen::Drifter::insert\("),
    ],
    "bdt_add.inc": [("gen/src/BinnedDiffusion_transform.cxx", r"^bool Gen::BinnedDiffusion_transform::add\(")],
}


def block(text, start):
    """The text from the first line matching ``start`` to the brace closing
    the first brace opened at or after it (and a ';' right after it)."""
    m = re.search(start, text, flags=re.M)
    if m is None:
        raise SystemExit("not found: " + start)
    i = m.start()
    depth, opened = 0, False
    for j in range(text.index("{", m.start()), len(text)):
        c = text[j]
        if c == "{":
            depth += 1
            opened = True
        elif c == "}":
            depth -= 1
            if opened and depth == 0:
                end = j + 1
                if text[end:end + 1] == ";":
                    end += 1
                return text[i:end] + "\n"
    raise SystemExit("unbalanced braces after: " + start)


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    for name, parts in PIECES.items():
        chunks = []
        for part in parts:
            path, start = part[0], part[1]
            with open(os.path.join(ref, path)) as f:
                text = f.read()
            if len(part) > 2 and part[2] == "rest":
                m = re.search(start, text, flags=re.M)
                if m is None:
                    raise SystemExit("not found: " + start)
                chunks.append("// %s\n" % path + text[m.start():])
            else:
                chunks.append("// %s\n" % path + block(text, start))
        with open(os.path.join(out, name), "w") as f:
            f.write("\n".join(chunks))


if __name__ == "__main__":
    main()
