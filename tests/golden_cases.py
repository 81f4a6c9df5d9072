"""The golden cases of CuboKit's single-slice pins (``tests/golden/*.npz``) as engine calls.

Each case carries the inputs of one ``SingleslicePtychography.reconstruct`` call of CuboKit's tests (file:line in the
case's ``source``) and the py4DSTEM outputs it is pinned to.  The metric and bound are the reference's:
``max|a - b| / max(1, max|b|) < 2e-6`` for the Double engine (``PtychographyTests.swift:28-31``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def gap(a, b):
    """``PtychographyTests.swift:28-31``: max abs difference over max(1, max |b|); a NaN fails."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    if a.shape != b.shape or not np.all(np.isfinite(a)):
        return np.inf
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def complex_gap(a, b):
    return max(gap(np.real(a), np.real(b)), gap(np.imag(a), np.imag(b)))


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _cx(z, key, shape):
    return (z[key + "_re"] + 1j * z[key + "_im"]).reshape(shape)


@dataclass
class Case:
    name: str
    source: str
    amplitudes: np.ndarray
    positions: np.ndarray
    object: np.ndarray
    probe: np.ndarray
    kwargs: dict
    expect_object: np.ndarray
    expect_probe: np.ndarray
    expect_errors: np.ndarray
    extra: dict = field(default_factory=dict)

    def result_gap(self, obj, probe, errors):
        return max(complex_gap(obj, self.expect_object), complex_gap(probe, self.expect_probe),
                   gap(errors, self.expect_errors))


def engine_cases():
    """Every single-slice engine pin of CuboKit's tests."""
    cases = []
    z = load("ptycho")
    R, C, OR, OC = (int(z[k]) for k in ("rows", "columns", "objectRows", "objectColumns"))
    probe = _cx(z, "initialProbe", (R, C))
    obj = _cx(z, "initialObject", (OR, OC))
    off = _cx(z, "offcentreProbe", (R, C))
    mean = dict(error_normalization="meanIntensity", mean_intensity=float(z["meanIntensity"]))
    amps = z["amplitudes"].reshape(-1, R, C)
    pos = z["positions"]
    cases.append(Case("ptycho.main", "PtychographyTests.swift:48-60", amps, pos, obj, probe,
                      dict(iterations=3, step_size=0.35, normalization_minimum=0.7, **mean),
                      _cx(z, "object", (OR, OC)), _cx(z, "probe", (R, C)), z["errors"]))
    for i in range(int(z["variants"])):
        v = lambda k: z[f"variant{i}_" + k]
        cases.append(Case(f"ptycho.variant{i}", "PtychographyTests.swift:61-70", amps, pos, obj, probe,
                          dict(iterations=3, step_size=float(v("step")), normalization_minimum=float(v("minimum")),
                               fix_probe=bool(v("fixProbe")), pure_phase_object=bool(v("purePhase")), **mean),
                          _cx(z, f"variant{i}_object", (OR, OC)), _cx(z, f"variant{i}_probe", (R, C)), v("errors")))
    for i in range(int(z["constraintCases"])):
        v = lambda k: z[f"constraint{i}_" + k]
        cases.append(Case(f"ptycho.constraint.{v('name')}", "PtychographyTests.swift:104-118", amps, pos, obj, off,
                          dict(iterations=3, step_size=0.35, normalization_minimum=0.7,
                               fix_probe_center_of_mass=bool(v("fixProbeCenterOfMass")),
                               constrain_probe_amplitude=bool(v("constrainProbeAmplitude")),
                               probe_amplitude_relative_radius=float(v("radius")),
                               probe_amplitude_relative_width=float(v("width")), **mean),
                          _cx(z, f"constraint{i}_object", (OR, OC)), _cx(z, f"constraint{i}_probe", (R, C)),
                          v("errors")))
    z = load("odd")
    R, C, OR, OC = (int(z[k]) for k in ("rows", "columns", "objectRows", "objectColumns"))
    probe = _cx(z, "startProbe", (R, C))
    obj = _cx(z, "initialObject", (OR, OC))
    mean = dict(error_normalization="meanIntensity", mean_intensity=float(z["meanIntensity"]))
    for i in range(int(z["cases"])):
        v = lambda k: z[f"case{i}_" + k]
        cases.append(Case(f"odd.{v('name')}", "OddSizeTests.swift:132-146", z["amplitudes"].reshape(-1, R, C),
                          z["positions"], obj, probe,
                          dict(iterations=3, step_size=0.35, normalization_minimum=0.7,
                               fix_probe_center_of_mass=bool(v("fixProbeCenterOfMass")),
                               constrain_probe_amplitude=bool(v("constrainProbeAmplitude")),
                               probe_amplitude_relative_radius=float(v("radius")),
                               probe_amplitude_relative_width=float(v("width")),
                               fix_probe_aperture=bool(v("aperture")),
                               probe_support_mask=z["support"].reshape(R, C) if bool(v("support")) else None, **mean),
                          _cx(z, f"case{i}_object", (OR, OC)), _cx(z, f"case{i}_probe", (R, C)), v("errors")))
    z = load("engines")
    R, C, OR, OC = (int(z[k]) for k in ("rows", "columns", "objectRows", "objectColumns"))
    probe = _cx(z, "startProbe", (R, C))
    obj = _cx(z, "initialObject", (OR, OC))
    mean = dict(error_normalization="meanIntensity", mean_intensity=float(z["meanIntensity"]))
    for i in range(int(z["cases"])):
        v = lambda k: z[f"case{i}_" + k]
        cases.append(Case(f"engines.{v('name')}", "EngineTests.swift:262-305", z["amplitudes"].reshape(-1, R, C),
                          z["positions"], obj, probe,
                          dict(iterations=3, step_size=0.35, normalization_minimum=0.7, fix_probe=bool(v("fixProbe")),
                               fix_probe_center_of_mass=bool(v("fixProbeCenterOfMass")),
                               constrain_probe_amplitude=bool(v("constrainProbeAmplitude")),
                               probe_amplitude_relative_radius=float(v("radius")),
                               probe_amplitude_relative_width=float(v("width")),
                               fix_probe_aperture=bool(v("fixProbeAperture")),
                               probe_support_mask=z["support"].reshape(R, C), **mean),
                          _cx(z, f"case{i}_object", (OR, OC)), _cx(z, f"case{i}_probe", (R, C)), v("errors")))
    p = load("ptycho")
    o = load("options")
    R, C, OR, OC = (int(p[k]) for k in ("rows", "columns", "objectRows", "objectColumns"))
    probe = _cx(p, "initialProbe", (R, C))
    start = _cx(o, "startObject", (OR, OC))
    mean = dict(error_normalization="meanIntensity", mean_intensity=float(p["meanIntensity"]))
    for i in range(int(o["amplitudeCases"])):
        v = lambda k: o[f"amp{i}_" + k]
        cases.append(Case(f"options.{v('name')}", "OptionsTests.swift:63-80", p["amplitudes"].reshape(-1, R, C),
                          p["positions"], start, probe,
                          dict(iterations=int(v("iterations")), step_size=float(v("step")), normalization_minimum=0.7,
                               fix_probe=bool(v("fixProbe")), pure_phase_object=bool(v("purePhase")),
                               constrain_object_amplitude=False, **mean),
                          _cx(o, f"amp{i}_object", (OR, OC)), _cx(o, f"amp{i}_probe", (R, C)), v("errors"),
                          extra=dict(maxAmplitude=float(v("maxAmplitude")))))
    return cases


def probe_cases():
    """Probe-builder pins: (name, kwargs of PtychographyProbe.build, expected probe)."""
    out = []
    z = load("ptycho")
    R, C = int(z["rows"]), int(z["columns"])
    wl = float(z["wavelength"])
    base = dict(row_sampling=0.8, column_sampling=1.1, wavelength=wl, cutoff=0.018, defocus=70, astigmatism=25,
                astigmatism_angle=0.31, spherical_aberration=2e4)
    out.append(("ptycho.builtProbe", dict(rows=R, columns=C, rolloff=0.002, **base), _cx(z, "builtProbe", (R, C))))
    out.append(("ptycho.rectangularProbe", dict(rows=7, columns=10, rolloff=0.0, **base),
                _cx(z, "rectangularProbe", (7, 10))))
    z = load("odd")
    R, C = int(z["rows"]), int(z["columns"])
    out.append(("odd.builtProbe", dict(rows=R, columns=C, row_sampling=float(z["rowSampling"]),
                                       column_sampling=float(z["columnSampling"]), wavelength=float(z["wavelength"]),
                                       cutoff=0.018, rolloff=0.002, defocus=70, astigmatism=25, astigmatism_angle=0.31,
                                       spherical_aberration=2e4), _cx(z, "builtProbe", (R, C))))
    o = load("options")
    g = lambda k: o["probes_" + k]
    R, C = int(g("rows")), int(g("columns"))
    for i in range(int(o["probeCases"])):
        v = lambda k: o[f"probe{i}_" + k]
        terms = []
        for n, m, mag, az in v("terms"):
            if int(m) == 0:
                terms.append((n, 0, 0.0, mag))
            else:
                terms.append((n, m, 0.0, mag * np.cos(m * az)))
                terms.append((n, m, 1.0, mag * np.sin(m * az)))
        out.append((f"options.{v('name')}", dict(rows=R, columns=C, row_sampling=float(g("rowSampling")),
                                                 column_sampling=float(g("columnSampling")),
                                                 wavelength=float(g("wavelength")), cutoff=float(g("cutoff")),
                                                 rolloff=float(g("rolloff")), defocus=float(v("defocus")),
                                                 astigmatism=float(v("astigmatism")),
                                                 astigmatism_angle=float(v("astigmatismAngle")),
                                                 spherical_aberration=float(v("sphericalAberration")),
                                                 terms=np.asarray(terms, np.float64).reshape(-1, 4)),
                    _cx(o, f"probe{i}_probe", (R, C))))
    for i in range(int(o["appCases"])):
        v = lambda k: o[f"app{i}_" + k]
        c12a, c12b = float(v("c12a")), float(v("c12b"))
        out.append((f"options.app.{v('name')}", dict(rows=R, columns=C, row_sampling=float(g("rowSampling")),
                                                     column_sampling=float(g("columnSampling")),
                                                     wavelength=float(g("wavelength")), cutoff=float(g("cutoff")),
                                                     rolloff=float(g("rolloff")), defocus=float(v("defocus")),
                                                     astigmatism=float(np.hypot(c12a, c12b)),
                                                     astigmatism_angle=float(0.5 * np.arctan2(c12b, c12a)),
                                                     terms=v("terms")), _cx(o, f"app{i}_probe", (R, C))))
    return out


def position_cases():
    """``PositionCorrectionTests.swift:43-62``: the five settings on the shared start, four iterations, step 0.35,
    normalisation minimum 0.7, mean-intensity errors.  Each entry: (name, inputs, settings, expected) with settings
    ``dict(step_size, max_update_distance, max_total_distance, row_sampling, column_sampling,
    constrain_center_of_mass)`` (distances in Å, None = unlimited) and expected ``(object, probe, errors, positions)``."""
    z = load("positions")
    R, C, OR, OC = int(z["rows"]), int(z["columns"]), int(z["objectRows"]), int(z["objectColumns"])
    base = dict(amplitudes=z["amplitudes"].reshape(-1, R, C), positions=z["nominalPositions"],
                obj=_cx(z, "startObject", (OR, OC)), probe=_cx(z, "startProbe", (R, C)), iterations=4, step_size=0.35,
                normalization_minimum=0.7, error_normalization="meanIntensity", mean_intensity=float(z["meanIntensity"]))
    out = []
    for name in z["cases"]:
        st = z[f"case_{name}_settings"]
        settings = dict(step_size=float(st[0]), max_update_distance=None if np.isnan(st[1]) else float(st[1]),
                        max_total_distance=None if np.isnan(st[2]) else float(st[2]),
                        row_sampling=float(z["rowSampling"]), column_sampling=float(z["columnSampling"]),
                        constrain_center_of_mass=bool(st[3]))
        inputs = dict(base, fix_probe=bool(z[f"case_{name}_fixProbe"]))
        expected = (_cx(z, f"case_{name}_object", (OR, OC)), _cx(z, f"case_{name}_probe", (R, C)),
                    z[f"case_{name}_errors"], z[f"case_{name}_positions"])
        out.append((str(name), inputs, settings, expected))
    return out


def position_exact_case():
    """``PositionCorrectionTests.swift:83-101``: exact object and probe, data taken at ``truthPositions``, the object
    frozen (step 1e-12), one iteration: the correction alone moves the positions."""
    z = load("positions")
    R, C, OR, OC = int(z["rows"]), int(z["columns"]), int(z["objectRows"]), int(z["objectColumns"])
    inputs = dict(amplitudes=z["exact_amplitudes"].reshape(-1, R, C), positions=z["nominalPositions"],
                  obj=_cx(z, "exact_object", (OR, OC)), probe=_cx(z, "exact_probe", (R, C)), iterations=1,
                  step_size=1e-12, normalization_minimum=0.7, fix_probe=True, error_normalization="meanIntensity",
                  mean_intensity=float(z["exact_meanIntensity"]))
    settings = dict(step_size=0.5, max_update_distance=None, max_total_distance=None, row_sampling=None,
                    column_sampling=None, constrain_center_of_mass=False)
    return inputs, settings, z["exact_positions"], z["truthPositions"], (float(z["rowSampling"]), float(z["columnSampling"]))


def align_phases(a, b):
    """Each state of ``a`` rotated by the global phase that best matches ``b`` (the eigenvector phase convention of the
    orthogonalisation is free; ``EngineTests.swift:46-64``)."""
    out = np.array(a, np.complex128)
    for s in range(out.shape[0]):
        z = np.sum(np.conj(b[s]) * out[s])
        if abs(z) > 0:
            out[s] = out[s] * np.conj(z) / abs(z)
    return out


def mixed_cases():
    """``EngineTests.swift:86-110``: five mixed-state settings on the shared start, three iterations, step 0.35,
    normalisation minimum 0.7, mean-intensity errors.  Each entry: (name, inputs, expected (object, probes, errors),
    orthogonalised)."""
    z = load("mixed")
    R, C, OR, OC = int(z["rows"]), int(z["columns"]), int(z["objectRows"]), int(z["objectColumns"])
    start = _cx(z, "startStates", (3, R, C))
    out = []
    for i in range(int(z["cases"])):
        g = lambda k: z[f"case{i}_{k}"]
        S = int(g("numProbes"))
        inputs = dict(amplitudes=z["amplitudes"].reshape(-1, R, C), positions=z["positions"],
                      obj=_cx(z, "initialObject", (OR, OC)), probes=start[:S], iterations=3, step_size=0.35,
                      normalization_minimum=0.7, fix_probe=bool(g("fixProbe")), pure_phase_object=bool(g("purePhase")),
                      fix_probe_center_of_mass=bool(g("fixProbeCenterOfMass")),
                      constrain_probe_amplitude=bool(g("constrainProbeAmplitude")),
                      probe_amplitude_relative_radius=float(g("radius")),
                      probe_amplitude_relative_width=float(g("width")), orthogonalize_probes=bool(g("orthogonalize")),
                      error_normalization="meanIntensity", mean_intensity=float(z["meanIntensity"]))
        expected = (_cx(z, f"case{i}_object", (OR, OC)), _cx(z, f"case{i}_probes", (S, R, C)), g("errors"))
        out.append((str(g("name")), inputs, expected, bool(g("orthogonalize"))))
    for i in range(int(z["extras"])):  # EngineTests.swift:262-305, the mixed engine's aperture / support cases
        g = lambda k: z[f"extra{i}_{k}"]
        inputs = dict(amplitudes=z["amplitudes"].reshape(-1, R, C), positions=z["positions"],
                      obj=_cx(z, "initialObject", (OR, OC)), probes=start[:2], iterations=3, step_size=0.35,
                      normalization_minimum=0.7, fix_probe=bool(g("fixProbe")),
                      fix_probe_center_of_mass=bool(g("fixProbeCenterOfMass")),
                      constrain_probe_amplitude=bool(g("constrainProbeAmplitude")),
                      probe_amplitude_relative_radius=float(g("radius")),
                      probe_amplitude_relative_width=float(g("width")), fix_probe_aperture=bool(g("fixProbeAperture")),
                      probe_support_mask=z["support"].reshape(R, C), error_normalization="meanIntensity",
                      mean_intensity=float(z["meanIntensity"]))
        expected = (_cx(z, f"extra{i}_object", (OR, OC)), _cx(z, f"extra{i}_probe", (2, R, C)), g("errors"))
        out.append(("extras." + str(g("name")), inputs, expected, True))
    return out


def mixed_orthogonalization_case():
    z = load("mixed")
    R, C = int(z["rows"]), int(z["columns"])
    count = int(z["orth_count"])
    return _cx(z, "orth_input", (count, R, C)), _cx(z, "orth_output", (count, R, C))


def mixed_init_cases():
    """``EngineTests.swift:131-149``: py4DSTEM's initial states (first state scaled to the mean intensity)."""
    z = load("mixed")
    R, C = int(z["rows"]), int(z["columns"])
    out = []
    for i in range(int(z["inits"])):
        g = lambda k: z[f"init{i}_{k}"]
        first = _cx(z, f"init{i}_first", (R, C))
        first = first * np.sqrt(float(g("meanIntensity")) / (np.sum(np.abs(first) ** 2) * R * C))
        count = int(g("count"))
        out.append((first, count, int(g("seed")), _cx(z, f"init{i}_states", (count, R, C)), g("draws")))
    return out


def multislice_cases():
    """``EngineTests.swift:205-228`` (six cases) and ``:262-305`` (the multislice engine's aperture / support extras):
    three iterations, step 0.35, normalisation minimum 0.7, mean-intensity errors.  Each entry: (name, inputs, expected
    (slices, probe, errors))."""
    z = load("multislice")
    R, C, OR, OC = int(z["rows"]), int(z["columns"]), int(z["objectRows"]), int(z["objectColumns"])
    start = _cx(z, "startSlices", (3, OR, OC))
    common = dict(amplitudes=z["amplitudes"].reshape(-1, R, C), positions=z["positions"],
                  probe=_cx(z, "startProbe", (R, C)), wavelength=float(z["wavelength"]),
                  row_sampling=float(z["rowSampling"]), column_sampling=float(z["columnSampling"]), iterations=3,
                  step_size=0.35, normalization_minimum=0.7, error_normalization="meanIntensity",
                  mean_intensity=float(z["meanIntensity"]))
    out = []
    for i in range(int(z["cases"])):
        g = lambda k: z[f"case{i}_{k}"]
        L = int(g("slices"))
        inputs = dict(common, obj=start[:L], slice_thicknesses=list(g("thicknesses")), fix_probe=bool(g("fixProbe")),
                      pure_phase_object=bool(g("purePhase")), identical_slices=bool(g("identicalSlices")),
                      fix_probe_center_of_mass=bool(g("fixProbeCenterOfMass")),
                      constrain_probe_amplitude=bool(g("constrainProbeAmplitude")),
                      probe_amplitude_relative_radius=float(g("radius")),
                      probe_amplitude_relative_width=float(g("width")))
        out.append((str(g("name")), inputs, (_cx(z, f"case{i}_object", (L, OR, OC)), _cx(z, f"case{i}_probe", (R, C)),
                                             g("errors"))))
    for i in range(int(z["extras"])):
        g = lambda k: z[f"extra{i}_{k}"]
        inputs = dict(common, obj=start[:3], slice_thicknesses=[55.0, 80.0], fix_probe=bool(g("fixProbe")),
                      fix_probe_center_of_mass=bool(g("fixProbeCenterOfMass")),
                      constrain_probe_amplitude=bool(g("constrainProbeAmplitude")),
                      probe_amplitude_relative_radius=float(g("radius")),
                      probe_amplitude_relative_width=float(g("width")), fix_probe_aperture=bool(g("fixProbeAperture")),
                      probe_support_mask=z["support"].reshape(R, C))
        out.append(("extras." + str(g("name")), inputs,
                    (_cx(z, f"extra{i}_object", (3, OR, OC)), _cx(z, f"extra{i}_probe", (R, C)), g("errors"))))
    return out


def multislice_propagator_case():
    z = load("multislice")
    R, C = int(z["rows"]), int(z["columns"])
    args = dict(rows=R, columns=C, row_sampling=float(z["rowSampling"]), column_sampling=float(z["columnSampling"]),
                wavelength=float(z["wavelength"]), slice_thicknesses=list(z["sliceThicknesses"]))
    return args, _cx(z, "propagators", (len(z["sliceThicknesses"]), R, C))
