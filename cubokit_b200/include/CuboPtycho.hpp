// CuboPtycho.hpp — C++ mirror of CuboPtycho's ptychography API over the B200 engine (include/cubo_ptycho.h).
//
// Names, argument meanings, defaults and error behaviour follow the Swift API (Sources/CuboPtycho/Ptychography.swift:
// PtychographyArray :5-21, PtychographyError :24-27, PtychographyErrorNormalization :30-48, PtychographyPosition :88-93,
// PtychographyAberrationTerm :101-133, PtychographyProbe.build :142-172, SingleslicePtychography.reconstruct
// :218-406 and its Result :179-188; PtychographyEngines.swift: PtychographyStack :13-27, MixedstatePtychography
// :121-330, MultislicePtychography :413-588).  Swift's labelled default arguments become the fields of each engine's
// Options, with the same defaults.  Refusals throw PtychographyError (invalidInput),
// cancellation throws CancellationError; device failures the CPU path cannot have throw DeviceError.
// Header-only; link with libcuboptycho.so.
#pragma once

#include <cmath>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cubo_ptycho.h"

namespace CuboPtycho {

// PtychographyError.invalidInput
struct PtychographyError : std::invalid_argument {
    explicit PtychographyError(const std::string &what) : std::invalid_argument("invalidInput: " + what) {}
};
struct CancellationError : std::runtime_error {
    CancellationError() : std::runtime_error("cancelled") {}
};
struct DeviceError : std::runtime_error {
    int status;
    DeviceError(int s, const std::string &what) : std::runtime_error(what), status(s) {}
};

// A finite row-major complex field in Double precision (Ptychography.swift:5-21).
struct PtychographyArray {
    int rows = 0, columns = 0;
    std::vector<double> real, imaginary;
    PtychographyArray(int rows_, int columns_, std::vector<double> real_, std::vector<double> imaginary_)
        : rows(rows_), columns(columns_), real(std::move(real_)), imaginary(std::move(imaginary_)) {
        const bool ok = rows > 1 && columns > 1 && (long long)rows * columns == (long long)real.size() &&
                        imaginary.size() == real.size();
        if (!ok) throw PtychographyError("array shape");
        for (size_t i = 0; i < real.size(); i++)
            if (!std::isfinite(real[i]) || !std::isfinite(imaginary[i])) throw PtychographyError("array not finite");
    }
};

// `count` finite complex grids of rows x columns, [index][row][column] (PtychographyEngines.swift:13-27): probe states
// or object slices.
struct PtychographyStack {
    int count = 0, rows = 0, columns = 0;
    std::vector<double> real, imaginary;
    PtychographyStack(int count_, int rows_, int columns_, std::vector<double> real_, std::vector<double> imaginary_)
        : count(count_), rows(rows_), columns(columns_), real(std::move(real_)), imaginary(std::move(imaginary_)) {
        const bool ok = count > 0 && rows > 1 && columns > 1 &&
                        (long long)count * rows * columns == (long long)real.size() && imaginary.size() == real.size();
        if (!ok) throw PtychographyError("stack shape");
        for (size_t i = 0; i < real.size(); i++)
            if (!std::isfinite(real[i]) || !std::isfinite(imaginary[i])) throw PtychographyError("stack not finite");
    }
};

struct PtychographyPosition {
    double row, column;
};

// How errors are normalised (Ptychography.swift:30-48).
struct PtychographyErrorNormalization {
    bool mean = false;
    double meanIntensityValue = 0;
    static PtychographyErrorNormalization meanIntensity(double m) { return {true, m}; }
    static PtychographyErrorNormalization suppliedAmplitudeEnergy() { return {false, 0}; }
};

// The GPU form; the reference's .double / .single become the FP64 and FP32 forms.
enum class PtychographyPrecision { fp32, splitBF16, fp64 };

// One aberration term beyond defocus, C12 and C30 (Ptychography.swift:101-133).
struct PtychographyAberrationTerm {
    enum class Component { cosine, sine };
    int radialOrder;
    int angularOrder;
    Component component;
    double coefficient;
    // py4DSTEM's polar C_nm cos(m (phi - phi_nm)) as Cartesian terms (Ptychography.swift:117-122)
    static std::vector<PtychographyAberrationTerm> polar(int n, int m, double magnitude, double azimuth) {
        if (m == 0) return {{n, 0, Component::cosine, magnitude}};
        return {{n, m, Component::cosine, magnitude * std::cos(m * azimuth)},
                {n, m, Component::sine, magnitude * std::sin(m * azimuth)}};
    }
};

// A device context; one per host thread (the engine's calls are blocking).
class Context {
  public:
    explicit Context(int device = 0) {
        const int st = cubo_ptycho_create(device, &ctx_);
        if (st != CUBO_PTYCHO_OK) throw DeviceError(st, "cubo_ptycho_create failed");
    }
    ~Context() { cubo_ptycho_destroy(ctx_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    cubo_ptycho_context *get() const { return ctx_; }
    void check(int status) const {
        if (status == CUBO_PTYCHO_OK) return;
        const std::string what = cubo_ptycho_last_error(ctx_);
        if (status == CUBO_PTYCHO_INVALID_INPUT) throw PtychographyError(what);
        if (status == CUBO_PTYCHO_CANCELLED) throw CancellationError();
        throw DeviceError(status, what);
    }
    static Context &shared(int device = 0) {
        static thread_local std::unique_ptr<Context> ctx;
        if (!ctx) ctx.reset(new Context(device));
        return *ctx;
    }

  private:
    cubo_ptycho_context *ctx_ = nullptr;
};

// PtychographyProbe.build (Ptychography.swift:142-172), evaluated on the device in FP64.
struct PtychographyProbe {
    static PtychographyArray build(int rows, int columns, double rowSampling, double columnSampling, double wavelength,
                                   double cutoff, double rolloff = 0.002, double defocus = 0, double astigmatism = 0,
                                   double astigmatismAngle = 0, double sphericalAberration = 0,
                                   const std::vector<PtychographyAberrationTerm> &higherOrder = {},
                                   Context &ctx = Context::shared()) {
        std::vector<double> terms;
        for (const auto &t : higherOrder) {
            terms.push_back(t.radialOrder);
            terms.push_back(t.angularOrder);
            terms.push_back(t.component == PtychographyAberrationTerm::Component::sine ? 1 : 0);
            terms.push_back(t.coefficient);
        }
        if (rows < 2 || columns < 2) throw PtychographyError("probe shape");
        std::vector<double> re((size_t)rows * columns), im((size_t)rows * columns);
        ctx.check(cubo_ptycho_probe_build(ctx.get(), rows, columns, rowSampling, columnSampling, wavelength, cutoff,
                                          rolloff, defocus, astigmatism, astigmatismAngle, sphericalAberration,
                                          (int)higherOrder.size(), terms.empty() ? nullptr : terms.data(), re.data(),
                                          im.data()));
        return PtychographyArray(rows, columns, std::move(re), std::move(im));
    }
};

// The labelled arguments of SingleslicePtychography.reconstruct(...) with their defaults (Ptychography.swift:218-234).
struct SingleslicePtychographyOptions {
    int iterations = 8;
    double stepSize = 0.5;
    double normalizationMinimum = 1;
    bool fixProbe = false;
    bool purePhaseObject = false;
    bool constrainObjectAmplitude = true;
    bool fixProbeCenterOfMass = false;
    bool constrainProbeAmplitude = false;
    double probeAmplitudeRelativeRadius = 0.5;
    double probeAmplitudeRelativeWidth = 0.05;
    bool fixProbeAperture = false;
    const std::vector<bool> *probeSupportMask = nullptr;
    PtychographyErrorNormalization errorNormalization = PtychographyErrorNormalization::suppliedAmplitudeEnergy();
    bool positionCorrection = false;  // refused on the GPU path, as .single refuses it (Ptychography.swift:236)
    PtychographyPrecision precision = PtychographyPrecision::fp32;
    int gatherTile = 0;  // object-gather tile choice (performance only), see cubo_ptycho_params.gather_tile
    int passShape = 0;   // position-pass CTA shape (performance only), see cubo_ptycho_params.pass_shape
    std::function<bool()> isCancelled;
    std::function<void(int, int)> progress;
};

struct SingleslicePtychography {
    // Result (Ptychography.swift:179-188)
    struct Result {
        PtychographyArray object;
        PtychographyArray probe;
        std::vector<double> errors;
        std::vector<PtychographyPosition> positions;
    };

    using Options = SingleslicePtychographyOptions;

    // Reconstructs from corner-centred Float32 amplitudes [position][row][column] (reconstructSingle's amplitude type,
    // PtychographySingle.swift:40-41; the Double overload converts as the reference's .single branch does).
    static Result reconstruct(const std::vector<float> &amplitudes, const std::vector<PtychographyPosition> &positions,
                              const PtychographyArray &object, const PtychographyArray &probe,
                              const Options &o = Options(), Context &ctx = Context::shared()) {
        const size_t n = (size_t)probe.rows * probe.columns;
        if (positions.empty() || amplitudes.size() != positions.size() * n) throw PtychographyError("amplitudes");
        if (o.probeSupportMask && o.probeSupportMask->size() != n) throw PtychographyError("probe support mask");
        std::vector<double> pr(positions.size()), pc(positions.size());
        for (size_t i = 0; i < positions.size(); i++) { pr[i] = positions[i].row; pc[i] = positions[i].column; }
        cubo_ptycho_problem problem{probe.rows, probe.columns, object.rows, object.columns, (int)positions.size(),
                                    amplitudes.data(), pr.data(), pc.data()};
        cubo_ptycho_params p;
        cubo_ptycho_params_default(&p);
        p.iterations = o.iterations;
        p.step_size = o.stepSize;
        p.normalization_minimum = o.normalizationMinimum;
        p.fix_probe = o.fixProbe;
        p.pure_phase_object = o.purePhaseObject;
        p.constrain_object_amplitude = o.constrainObjectAmplitude;
        p.fix_probe_center_of_mass = o.fixProbeCenterOfMass;
        p.constrain_probe_amplitude = o.constrainProbeAmplitude;
        p.probe_amplitude_relative_radius = o.probeAmplitudeRelativeRadius;
        p.probe_amplitude_relative_width = o.probeAmplitudeRelativeWidth;
        p.fix_probe_aperture = o.fixProbeAperture;
        std::vector<unsigned char> mask;
        if (o.probeSupportMask) {
            for (bool b : *o.probeSupportMask) mask.push_back(b ? 1 : 0);
            p.probe_support_mask = mask.data();
        }
        p.error_normalization = o.errorNormalization.mean ? CUBO_PTYCHO_ERRORS_MEAN_INTENSITY
                                                          : CUBO_PTYCHO_ERRORS_SUPPLIED_AMPLITUDE_ENERGY;
        p.mean_intensity = o.errorNormalization.meanIntensityValue;
        p.has_position_correction = o.positionCorrection;
        p.gather_tile = o.gatherTile;
        p.pass_shape = o.passShape;
        p.form = o.precision == PtychographyPrecision::fp64        ? CUBO_PTYCHO_FORM_FP64
                 : o.precision == PtychographyPrecision::splitBF16 ? CUBO_PTYCHO_FORM_SPLIT_BF16
                                                                   : CUBO_PTYCHO_FORM_FP32;
        // isCancelled before every iteration, progress after each (Ptychography.swift:281,401)
        if (o.isCancelled && o.isCancelled()) throw CancellationError();
        struct Hooks {
            const Options *o;
            volatile int cancel;
        } hooks{&o, 0};
        if (o.isCancelled || o.progress) {
            p.cancel = &hooks.cancel;
            p.progress_user = &hooks;
            p.progress = [](int done, int total, void *user) {
                auto *h = static_cast<Hooks *>(user);
                if (h->o->progress) h->o->progress(done, total);
                if (h->o->isCancelled && h->o->isCancelled()) h->cancel = 1;
            };
        }
        std::vector<double> ore = object.real, oim = object.imaginary, pre = probe.real, pim = probe.imaginary;
        std::vector<double> errors(o.iterations > 0 ? o.iterations : 1);
        ctx.check(cubo_ptycho_reconstruct(ctx.get(), &problem, &p, ore.data(), oim.data(), pre.data(), pim.data(),
                                          errors.data()));
        errors.resize(o.iterations > 0 ? o.iterations : 0);
        return Result{PtychographyArray(object.rows, object.columns, std::move(ore), std::move(oim)),
                      PtychographyArray(probe.rows, probe.columns, std::move(pre), std::move(pim)), std::move(errors),
                      positions};
    }

    // The Double overload: amplitudes converted to Float after the reference's finite/non-negative check
    // (Ptychography.swift:237-239).
    static Result reconstruct(const std::vector<double> &amplitudes, const std::vector<PtychographyPosition> &positions,
                              const PtychographyArray &object, const PtychographyArray &probe,
                              const Options &o = Options(), Context &ctx = Context::shared()) {
        std::vector<float> f(amplitudes.size());
        for (size_t i = 0; i < amplitudes.size(); i++) {
            if (!(std::isfinite(amplitudes[i]) && amplitudes[i] >= 0)) throw PtychographyError("amplitude");
            f[i] = (float)amplitudes[i];
        }
        return reconstruct(f, positions, object, probe, o, ctx);
    }
};

namespace detail {

// The arguments every engine shares, as the C ABI takes them (the FP64 form: the engines are the reference's Double
// ones).  `mask` keeps the support mask's bytes alive for the call.
template <typename Options>
cubo_ptycho_params engine_params(const Options &o, size_t n, std::vector<unsigned char> &mask) {
    cubo_ptycho_params p;
    cubo_ptycho_params_default(&p);
    p.iterations = o.iterations;
    p.step_size = o.stepSize;
    p.normalization_minimum = o.normalizationMinimum;
    p.fix_probe = o.fixProbe;
    p.pure_phase_object = o.purePhaseObject;
    p.constrain_object_amplitude = 1;  // the engines always apply the threshold
    p.fix_probe_center_of_mass = o.fixProbeCenterOfMass;
    p.constrain_probe_amplitude = o.constrainProbeAmplitude;
    p.probe_amplitude_relative_radius = o.probeAmplitudeRelativeRadius;
    p.probe_amplitude_relative_width = o.probeAmplitudeRelativeWidth;
    p.fix_probe_aperture = o.fixProbeAperture;
    if (o.probeSupportMask) {
        if (o.probeSupportMask->size() != n) throw PtychographyError("probe support mask");
        for (bool b : *o.probeSupportMask) mask.push_back(b ? 1 : 0);
        p.probe_support_mask = mask.data();
    }
    p.error_normalization = o.errorNormalization.mean ? CUBO_PTYCHO_ERRORS_MEAN_INTENSITY
                                                      : CUBO_PTYCHO_ERRORS_SUPPLIED_AMPLITUDE_ENERGY;
    p.mean_intensity = o.errorNormalization.meanIntensityValue;
    p.form = CUBO_PTYCHO_FORM_FP64;
    return p;
}

inline cubo_ptycho_problem engine_problem(const std::vector<float> &amplitudes,
                                          const std::vector<PtychographyPosition> &positions, int rows, int columns,
                                          int object_rows, int object_columns, std::vector<double> &pr,
                                          std::vector<double> &pc) {
    const size_t n = (size_t)rows * columns;
    if (positions.empty() || amplitudes.size() != positions.size() * n) throw PtychographyError("amplitudes");
    pr.resize(positions.size());
    pc.resize(positions.size());
    for (size_t i = 0; i < positions.size(); i++) { pr[i] = positions[i].row; pc[i] = positions[i].column; }
    return cubo_ptycho_problem{rows, columns, object_rows, object_columns, (int)positions.size(), amplitudes.data(),
                               pr.data(), pc.data(), 0};
}

}  // namespace detail

// MixedstateZeroPixelError (PtychographyEngines.swift:4-10)
enum class MixedstateZeroPixelError { reference, finite };

// The labelled arguments of MixedstatePtychography.reconstruct(...) with their defaults (PtychographyEngines.swift:
// 148-157).
struct MixedstatePtychographyOptions {
    int iterations = 8;
    double stepSize = 0.5;
    double normalizationMinimum = 1;
    bool fixProbe = false;
    bool purePhaseObject = false;
    bool fixProbeCenterOfMass = false;
    bool constrainProbeAmplitude = false;
    double probeAmplitudeRelativeRadius = 0.5;
    double probeAmplitudeRelativeWidth = 0.05;
    bool orthogonalizeProbes = true;
    bool fixProbeAperture = false;
    const std::vector<bool> *probeSupportMask = nullptr;
    PtychographyErrorNormalization errorNormalization = PtychographyErrorNormalization::suppliedAmplitudeEnergy();
    MixedstateZeroPixelError zeroFarFieldPixelError = MixedstateZeroPixelError::reference;
};

// MixedstatePtychography (PtychographyEngines.swift:121-330): several incoherent probe states on one object, FP64.
struct MixedstatePtychography {
    struct Result {  // :126-134
        PtychographyArray object;
        PtychographyStack probes;
        std::vector<double> errors;
    };
    using Options = MixedstatePtychographyOptions;

    static Result reconstruct(const std::vector<float> &amplitudes, const std::vector<PtychographyPosition> &positions,
                              const PtychographyArray &object, const PtychographyStack &probes,
                              const Options &o = Options(), Context &ctx = Context::shared()) {
        std::vector<double> pr, pc;
        std::vector<unsigned char> mask;
        cubo_ptycho_problem problem = detail::engine_problem(amplitudes, positions, probes.rows, probes.columns,
                                                             object.rows, object.columns, pr, pc);
        cubo_ptycho_params p = detail::engine_params(o, (size_t)probes.rows * probes.columns, mask);
        cubo_ptycho_mixed_params m;
        cubo_ptycho_mixed_params_default(&m);
        m.states = probes.count;
        m.orthogonalize_probes = o.orthogonalizeProbes;
        m.zero_pixel_error = o.zeroFarFieldPixelError == MixedstateZeroPixelError::reference
                                 ? CUBO_PTYCHO_ZERO_PIXEL_REFERENCE : CUBO_PTYCHO_ZERO_PIXEL_FINITE;
        std::vector<double> ore = object.real, oim = object.imaginary, pre = probes.real, pim = probes.imaginary;
        std::vector<double> errors(o.iterations > 0 ? o.iterations : 1);
        ctx.check(cubo_ptycho_mixed_reconstruct(ctx.get(), &problem, &p, &m, ore.data(), oim.data(), pre.data(),
                                                pim.data(), errors.data()));
        errors.resize(o.iterations > 0 ? o.iterations : 0);
        return Result{PtychographyArray(object.rows, object.columns, std::move(ore), std::move(oim)),
                      PtychographyStack(probes.count, probes.rows, probes.columns, std::move(pre), std::move(pim)),
                      std::move(errors)};
    }

    // MixedstatePtychography.orthogonalize (:265-269): the eigenvectors of the states' Gram matrix, by decreasing
    // intensity (each state's overall phase is free).
    static PtychographyStack orthogonalize(const PtychographyStack &probes, Context &ctx = Context::shared()) {
        std::vector<double> re = probes.real, im = probes.imaginary;
        ctx.check(cubo_ptycho_orthogonalize(ctx.get(), probes.count, probes.rows, probes.columns, re.data(), im.data()));
        return PtychographyStack(probes.count, probes.rows, probes.columns, std::move(re), std::move(im));
    }
};

// The labelled arguments of MultislicePtychography.reconstruct(...) after the geometry, with their defaults
// (PtychographyEngines.swift:454-462).
struct MultislicePtychographyOptions {
    int iterations = 8;
    double stepSize = 0.5;
    double normalizationMinimum = 1;
    bool fixProbe = false;
    bool purePhaseObject = false;
    bool identicalSlices = false;
    bool fixProbeCenterOfMass = false;
    bool constrainProbeAmplitude = false;
    double probeAmplitudeRelativeRadius = 0.5;
    double probeAmplitudeRelativeWidth = 0.05;
    bool fixProbeAperture = false;
    const std::vector<bool> *probeSupportMask = nullptr;
    PtychographyErrorNormalization errorNormalization = PtychographyErrorNormalization::suppliedAmplitudeEnergy();
};

// MultislicePtychography (PtychographyEngines.swift:413-588): object slices with Fresnel propagation between them, FP64.
struct MultislicePtychography {
    struct Result {  // :417-424
        PtychographyStack object;
        PtychographyArray probe;
        std::vector<double> errors;
    };
    using Options = MultislicePtychographyOptions;

    // MultislicePtychography.propagators (:427-442), host arithmetic.
    static PtychographyStack propagators(int rows, int columns, double rowSampling, double columnSampling,
                                         double wavelength, const std::vector<double> &sliceThicknesses) {
        const size_t size = sliceThicknesses.size() * (size_t)(rows > 0 ? rows : 0) * (size_t)(columns > 0 ? columns : 0);
        std::vector<double> re(size), im(size);
        const int st = cubo_ptycho_propagators(rows, columns, rowSampling, columnSampling, wavelength,
                                               (int)sliceThicknesses.size(),
                                               sliceThicknesses.empty() ? nullptr : sliceThicknesses.data(), re.data(),
                                               im.data());
        if (st != CUBO_PTYCHO_OK) throw PtychographyError("propagators");
        return PtychographyStack((int)sliceThicknesses.size(), rows, columns, std::move(re), std::move(im));
    }

    static Result reconstruct(const std::vector<float> &amplitudes, const std::vector<PtychographyPosition> &positions,
                              const PtychographyStack &object, const PtychographyArray &probe,
                              const std::vector<double> &sliceThicknesses, double wavelength, double rowSampling,
                              double columnSampling, const Options &o = Options(), Context &ctx = Context::shared()) {
        if ((int)sliceThicknesses.size() != object.count - 1) throw PtychographyError("slice thicknesses");
        std::vector<double> pr, pc;
        std::vector<unsigned char> mask;
        cubo_ptycho_problem problem = detail::engine_problem(amplitudes, positions, probe.rows, probe.columns,
                                                             object.rows, object.columns, pr, pc);
        cubo_ptycho_params p = detail::engine_params(o, (size_t)probe.rows * probe.columns, mask);
        cubo_ptycho_multislice_params m{object.count, sliceThicknesses.empty() ? nullptr : sliceThicknesses.data(),
                                        wavelength, rowSampling, columnSampling, o.identicalSlices ? 1 : 0};
        std::vector<double> ore = object.real, oim = object.imaginary, pre = probe.real, pim = probe.imaginary;
        std::vector<double> errors(o.iterations > 0 ? o.iterations : 1);
        ctx.check(cubo_ptycho_multislice_reconstruct(ctx.get(), &problem, &p, &m, ore.data(), oim.data(), pre.data(),
                                                     pim.data(), errors.data()));
        errors.resize(o.iterations > 0 ? o.iterations : 0);
        return Result{PtychographyStack(object.count, object.rows, object.columns, std::move(ore), std::move(oim)),
                      PtychographyArray(probe.rows, probe.columns, std::move(pre), std::move(pim)), std::move(errors)};
    }
};

}  // namespace CuboPtycho
