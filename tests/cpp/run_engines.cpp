// Runs one mixed-state or multislice reconstruction through the C++ mirror (cubokit_b200/include/CuboPtycho.hpp) on
// inputs written by tests/test_gpu_cpp.py and writes the results back for it to compare with CuboKit's pins.
//
//   run_engines mixed|multislice <in.bin> <out.bin>
//
// in (mixed):      int32 R, C, OR, OC, P, S, iterations, fixProbe, purePhase, centreOfMass, constrainAmplitude,
//                  orthogonalize; float64 step, minimum, meanIntensity, radius, width; amplitudes P*R*C, positions 2P,
//                  object re, im (OR*OC each), probes re, im (S*R*C each)
// in (multislice): int32 R, C, OR, OC, P, L, iterations, fixProbe, purePhase, identicalSlices, centreOfMass,
//                  constrainAmplitude; float64 step, minimum, meanIntensity, radius, width, wavelength, rowSampling,
//                  columnSampling; thicknesses L-1, amplitudes P*R*C, positions 2P, object re, im (L*OR*OC each),
//                  probe re, im (R*C each)
// out: float64 object re, im, probe(s) re, im, errors
#include <cstdio>
#include <string>
#include <vector>

#include "CuboPtycho.hpp"

namespace {

struct Reader {
    FILE *f;
    template <typename T> std::vector<T> take(size_t count) {
        std::vector<T> v(count);
        if (count && fread(v.data(), sizeof(T), count, f) != count) throw std::runtime_error("short input");
        return v;
    }
};

void put(FILE *f, const std::vector<double> &v) { fwrite(v.data(), sizeof(double), v.size(), f); }

}  // namespace

int main(int argc, char **argv) {
    using namespace CuboPtycho;
    if (argc != 4) return 2;
    const std::string which = argv[1];
    FILE *in = fopen(argv[2], "rb");
    if (!in) return 2;
    Reader r{in};
    try {
        const auto i = r.take<int32_t>(12);
        const int R = i[0], C = i[1], OR = i[2], OC = i[3], P = i[4], K = i[5];
        const size_t n = (size_t)R * C;
        std::vector<double> d = r.take<double>(which == "mixed" ? 5 : 8);
        std::vector<double> thick;
        if (which == "multislice") thick = r.take<double>(K - 1);
        const auto amp = r.take<double>((size_t)P * n);
        const auto pos = r.take<double>((size_t)2 * P);
        std::vector<float> amplitudes(amp.begin(), amp.end());
        std::vector<PtychographyPosition> positions(P);
        for (int k = 0; k < P; k++) positions[k] = {pos[2 * k], pos[2 * k + 1]};
        FILE *out = fopen(argv[3], "wb");
        if (!out) return 2;
        if (which == "mixed") {
            auto ore = r.take<double>((size_t)OR * OC), oim = r.take<double>((size_t)OR * OC);
            auto pre = r.take<double>(K * n), pim = r.take<double>(K * n);
            MixedstatePtychography::Options o;
            o.iterations = i[6];
            o.fixProbe = i[7];
            o.purePhaseObject = i[8];
            o.fixProbeCenterOfMass = i[9];
            o.constrainProbeAmplitude = i[10];
            o.orthogonalizeProbes = i[11];
            o.stepSize = d[0];
            o.normalizationMinimum = d[1];
            o.errorNormalization = PtychographyErrorNormalization::meanIntensity(d[2]);
            o.probeAmplitudeRelativeRadius = d[3];
            o.probeAmplitudeRelativeWidth = d[4];
            const auto res = MixedstatePtychography::reconstruct(
                amplitudes, positions, PtychographyArray(OR, OC, ore, oim), PtychographyStack(K, R, C, pre, pim), o);
            put(out, res.object.real);
            put(out, res.object.imaginary);
            put(out, res.probes.real);
            put(out, res.probes.imaginary);
            put(out, res.errors);
        } else {
            auto ore = r.take<double>((size_t)K * OR * OC), oim = r.take<double>((size_t)K * OR * OC);
            auto pre = r.take<double>(n), pim = r.take<double>(n);
            MultislicePtychography::Options o;
            o.iterations = i[6];
            o.fixProbe = i[7];
            o.purePhaseObject = i[8];
            o.identicalSlices = i[9];
            o.fixProbeCenterOfMass = i[10];
            o.constrainProbeAmplitude = i[11];
            o.stepSize = d[0];
            o.normalizationMinimum = d[1];
            o.errorNormalization = PtychographyErrorNormalization::meanIntensity(d[2]);
            o.probeAmplitudeRelativeRadius = d[3];
            o.probeAmplitudeRelativeWidth = d[4];
            const auto res = MultislicePtychography::reconstruct(
                amplitudes, positions, PtychographyStack(K, OR, OC, ore, oim), PtychographyArray(R, C, pre, pim), thick,
                d[5], d[6], d[7], o);
            put(out, res.object.real);
            put(out, res.object.imaginary);
            put(out, res.probe.real);
            put(out, res.probe.imaginary);
            put(out, res.errors);
        }
        fclose(out);
    } catch (const std::exception &e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    fclose(in);
    return 0;
}
