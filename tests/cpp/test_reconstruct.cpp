// C++ parity program for CuboPtycho.hpp, in the shape of CuboKit's PtychographyTests.threeIterationsAgainstSingleslice
// (Tests/CuboPtychoTests/PtychographyTests.swift:48-72): decode a pinned case, reconstruct, compare with the reference's
// gap metric (max |a - b| / max(1, max |b|), a NaN fails) against 2e-6.  Also the refusals (:73-85) and progress and
// cancellation (SinglePrecisionTests.swift:89-101).  The case file is written by tests/test_gpu_cpp.py.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <vector>

#include "CuboPtycho.hpp"

using namespace CuboPtycho;

static double gap(const std::vector<double> &a, const std::vector<double> &b) {
    if (a.size() != b.size()) return INFINITY;
    double m = 0, s = 1;
    for (size_t i = 0; i < a.size(); i++) {
        if (!std::isfinite(a[i])) return INFINITY;
        m = std::fmax(m, std::fabs(a[i] - b[i]));
        s = std::fmax(s, std::fabs(b[i]));
    }
    return m / s;
}

template <typename T> static std::vector<T> read(std::ifstream &f, size_t count) {
    std::vector<T> v(count);
    f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(count * sizeof(T)));
    return v;
}

int main(int argc, char **argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: test_reconstruct CASE\n"); return 2; }
    std::ifstream f(argv[1], std::ios::binary);
    const auto h = read<int32_t>(f, 6);  // rows, columns, objectRows, objectColumns, count, iterations
    const auto d = read<double>(f, 3);   // step, minimum, meanIntensity
    const int R = h[0], C = h[1], OR = h[2], OC = h[3], P = h[4], it = h[5];
    const size_t n = (size_t)R * C, no = (size_t)OR * OC;
    const auto amps = read<double>(f, P * n);
    const auto pos = read<double>(f, 2 * (size_t)P);
    const auto o_re = read<double>(f, no), o_im = read<double>(f, no);
    const auto p_re = read<double>(f, n), p_im = read<double>(f, n);
    const auto eo_re = read<double>(f, no), eo_im = read<double>(f, no);
    const auto ep_re = read<double>(f, n), ep_im = read<double>(f, n);
    const auto e_err = read<double>(f, it);
    if (!f) { std::fprintf(stderr, "short case file\n"); return 2; }
    std::vector<PtychographyPosition> positions;
    for (int i = 0; i < P; i++) positions.push_back({pos[2 * i], pos[2 * i + 1]});
    const PtychographyArray initialObject(OR, OC, o_re, o_im), initialProbe(R, C, p_re, p_im);
    int failures = 0;

    SingleslicePtychography::Options o;
    o.iterations = it;
    o.stepSize = d[0];
    o.normalizationMinimum = d[1];
    o.errorNormalization = PtychographyErrorNormalization::meanIntensity(d[2]);
    o.precision = PtychographyPrecision::fp64;
    const auto r = SingleslicePtychography::reconstruct(amps, positions, initialObject, initialProbe, o);
    double g = 0;
    for (double x : {gap(r.object.real, eo_re), gap(r.object.imaginary, eo_im), gap(r.probe.real, ep_re),
                     gap(r.probe.imaginary, ep_im), gap(r.errors, e_err)})
        g = std::fmax(g, x);
    std::printf("PTYCHO engine max normwise gap (fp64 form): %.3e\n", g);
    if (!(g < 2e-6)) failures++;

    o.precision = PtychographyPrecision::fp32;
    const auto r32 = SingleslicePtychography::reconstruct(amps, positions, initialObject, initialProbe, o);
    const double g32 = std::fmax(gap(r32.object.real, r.object.real), gap(r32.object.imaginary, r.object.imaginary));
    std::printf("fp32 form vs fp64 form, object: %.3e\n", g32);
    if (!(g32 < 1e-4)) failures++;

    // refusals: no positions; a probe-amplitude radius out of range (PtychographyTests.swift:73-85,172-180)
    try {
        SingleslicePtychography::reconstruct(std::vector<float>{}, {}, initialProbe, initialProbe);
        failures++;
    } catch (const PtychographyError &) {}
    try {
        SingleslicePtychography::Options bad = o;
        bad.constrainProbeAmplitude = true;
        bad.probeAmplitudeRelativeRadius = 0.51;
        SingleslicePtychography::reconstruct(amps, positions, initialObject, initialProbe, bad);
        failures++;
    } catch (const PtychographyError &) {}
    // progress [1, 2]; cancellation after the third poll
    std::vector<int> seen;
    SingleslicePtychography::Options pr = o;
    pr.iterations = 2;
    pr.progress = [&](int done, int total) { if (total == 2) seen.push_back(done); };
    SingleslicePtychography::reconstruct(amps, positions, initialObject, initialProbe, pr);
    if (seen != std::vector<int>{1, 2}) failures++;
    int polls = 0;
    SingleslicePtychography::Options cn = o;
    cn.iterations = 5;
    cn.isCancelled = [&] { return ++polls > 3; };
    try {
        SingleslicePtychography::reconstruct(amps, positions, initialObject, initialProbe, cn);
        failures++;
    } catch (const CancellationError &) {}
    std::printf("%s (%d failures)\n", failures ? "FAIL" : "OK", failures);
    return failures ? 1 : 0;
}
