"""Extract the single-slice ptychography golden vectors from CuboKit's committed py4DSTEM pins.

The pins are the JSON fixtures of CuboKit's own test suite (``Tests/CuboPtychoTests/Fixtures``), written by
``tools/ptycho/{pins,odd_pins,engines_pins,options_pins}.py`` from py4DSTEM f050d207 / 0.14.19.  This script keeps only
the fields the single-slice gradient-descent engine and the probe builder need and stores them as compressed ``.npz``
files beside itself, so the tests (which also run where the CuboKit checkout is absent) read plain arrays.

Run once, in a container that has the CuboKit checkout:  python tests/golden/make_golden.py CUBOKIT_ROOT

Which reference test each group pins (paths inside the CuboKit project):
  ptycho.npz   Tests/CuboPtychoTests/PtychographyTests.swift:33-72,104-118 (engine, variants, constraints, probe build)
  odd.npz      Tests/CuboPtychoTests/OddSizeTests.swift:122-146 (15x13 probe on a 31x29 object, single-slice cases)
  engines.npz  Tests/CuboPtychoTests/EngineTests.swift:262-305 (aperture / support extras, single-slice engine only)
  options.npz  Tests/CuboPtychoTests/OptionsTests.swift:48-145 (object amplitude toggle, higher-order probe terms)
  preprocess.npz  Tests/CuboPtychoTests/PreparationTests.swift:39-81 (pattern shifts, square-root amplitudes, mean
                  intensities: bilinear and cubic-spline orders, per-position origins)
  ptycho.npz also keeps the raw cube and uniform origin of PtychographyTests.swift:184-193 (bilinear preprocessing
                  through to the engine's amplitude pin)
  mixed.npz    Tests/CuboPtychoTests/EngineTests.swift:86-188,262-305 (mixed-state engine: five cases, the
                orthogonalisation, py4DSTEM's initial states, the mixed engine's support / aperture extras)
  multislice.npz  Tests/CuboPtychoTests/EngineTests.swift:190-255,262-305 (multislice engine: propagators, six
                  cases, the multislice engine's support / aperture extras)
  positions.npz  Tests/CuboPtychoTests/PositionCorrectionTests.swift:43-110 (position correction: five settings on
                  8 x 8 positions started up to 0.3 px off, four iterations; the exact-data case; tools/ptycho/
                  position_pins.py, py4DSTEM reconstruct(fix_positions=False))
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _cx(store, key, c):
    store[key + "_re"] = np.asarray(c["real"], np.float64)
    store[key + "_im"] = np.asarray(c["imaginary"], np.float64)


def _scalar(store, key, v):
    store[key] = np.asarray(v)


def ptycho(fx):
    p = json.loads((fx / "ptycho.json").read_text())
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns", "wavelength"):
        _scalar(s, k, p[k])
    s["positions"] = np.asarray(p["positions"], np.float64)
    s["amplitudes"] = np.asarray(p["amplitudes"], np.float64)
    _scalar(s, "meanIntensity", p["preprocessing"]["meanIntensity"])
    s["preprocessing_raw"] = np.asarray(p["preprocessing"]["raw"], np.float64)
    s["preprocessing_origin"] = np.asarray(p["preprocessing"]["origin"], np.float64)
    for k in ("initialProbe", "initialObject", "builtProbe", "object", "probe", "rectangularProbe", "offcentreProbe"):
        _cx(s, k, p[k])
    s["errors"] = np.asarray(p["errors"], np.float64)
    _scalar(s, "variants", len(p["variants"]))
    for i, v in enumerate(p["variants"]):
        pre = f"variant{i}_"
        for k in ("fixProbe", "purePhase", "minimum", "step"):
            _scalar(s, pre + k, v[k])
        _cx(s, pre + "object", v["object"])
        _cx(s, pre + "probe", v["probe"])
        s[pre + "errors"] = np.asarray(v["errors"], np.float64)
    _scalar(s, "constraintCases", len(p["constraintCases"]))
    for i, c in enumerate(p["constraintCases"]):
        pre = f"constraint{i}_"
        _scalar(s, pre + "name", c["name"])
        for k in ("fixProbeCenterOfMass", "constrainProbeAmplitude", "radius", "width"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    return s


def odd(fx):
    e = json.loads((fx / "odd.json").read_text())["engines"]
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns", "rowSampling", "columnSampling", "wavelength"):
        _scalar(s, k, e[k])
    s["positions"] = np.asarray(e["positions"], np.float64)
    s["amplitudes"] = np.asarray(e["amplitudes"], np.float64)
    s["support"] = np.asarray(e["support"], np.bool_)
    _scalar(s, "meanIntensity", e["multislicePreprocessing"]["meanIntensity"])
    _cx(s, "initialObject", e["initialObject"])
    _cx(s, "startProbe", e["startProbe"])
    _cx(s, "builtProbe", e["builtProbe"])
    _scalar(s, "cases", len(e["single"]))
    for i, c in enumerate(e["single"]):
        pre = f"case{i}_"
        _scalar(s, pre + "name", c["name"])
        for k in ("fixProbeCenterOfMass", "constrainProbeAmplitude", "radius", "width", "aperture", "support"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    return s


def engines(fx):
    p = json.loads((fx / "engines.json").read_text())
    m, x = p["multislice"], p["extras"]
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns"):
        _scalar(s, k, p[k])
    s["positions"] = np.asarray(p["positions"], np.float64)
    s["amplitudes"] = np.asarray(m["amplitudes"], np.float64)
    _scalar(s, "meanIntensity", m["preprocessing"]["meanIntensity"])
    _cx(s, "initialObject", p["initialObject"])
    _cx(s, "startProbe", m["startProbe"])
    s["support"] = np.asarray(x["support"], np.bool_)
    single = [c for c in x["cases"] if c["engine"] == "single"]
    _scalar(s, "cases", len(single))
    for i, c in enumerate(single):
        pre = f"case{i}_"
        _scalar(s, pre + "name", c["name"])
        for k in ("fixProbeCenterOfMass", "fixProbeAperture", "fixProbe", "constrainProbeAmplitude", "radius", "width"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    return s


def mixed(fx):
    """The mixed-state part of engines.json: reconstruction cases, the orthogonalisation pin, the initial states, and the
    mixed engine's support / aperture extras."""
    p = json.loads((fx / "engines.json").read_text())
    m, x = p["mixed"], p["extras"]
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns"):
        _scalar(s, k, p[k])
    s["positions"] = np.asarray(p["positions"], np.float64)
    _cx(s, "initialObject", p["initialObject"])
    s["amplitudes"] = np.asarray(m["amplitudes"], np.float64)
    _scalar(s, "meanIntensity", m["preprocessing"]["meanIntensity"])
    s["preprocessing_raw"] = np.asarray(m["preprocessing"]["raw"], np.float64)
    s["preprocessing_origin"] = np.asarray(m["preprocessing"]["origin"], np.float64)
    _cx(s, "startStates", m["startStates"])
    _scalar(s, "cases", len(m["cases"]))
    for i, c in enumerate(m["cases"]):
        pre = f"case{i}_"
        for k in ("name", "numProbes", "fixProbeCenterOfMass", "orthogonalize", "constrainProbeAmplitude", "radius",
                  "width", "fixProbe", "purePhase"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probes", c["probes"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    o = m["orthogonalization"]
    _scalar(s, "orth_count", o["count"])
    _cx(s, "orth_input", o["input"])
    _cx(s, "orth_output", o["output"])
    _scalar(s, "inits", len(m["inits"]))
    for i, c in enumerate(m["inits"]):
        pre = f"init{i}_"
        for k in ("seed", "count", "meanIntensity"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "first", c["first"])
        _cx(s, pre + "states", c["states"])
        s[pre + "draws"] = np.asarray(c["draws"], np.float64)
    s["support"] = np.asarray(x["support"], np.bool_)
    extras = [c for c in x["cases"] if c["engine"] == "mixed"]
    _scalar(s, "extras", len(extras))
    for i, c in enumerate(extras):
        pre = f"extra{i}_"
        _scalar(s, pre + "name", c["name"])
        for k in ("fixProbeCenterOfMass", "fixProbeAperture", "fixProbe", "constrainProbeAmplitude", "radius", "width"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    return s


def multislice(fx):
    """The multislice part of engines.json: propagators, reconstruction cases and the multislice engine's support /
    aperture extras."""
    p = json.loads((fx / "engines.json").read_text())
    m, x = p["multislice"], p["extras"]
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns", "rowSampling", "columnSampling", "wavelength"):
        _scalar(s, k, p[k])
    s["positions"] = np.asarray(p["positions"], np.float64)
    s["amplitudes"] = np.asarray(m["amplitudes"], np.float64)
    _scalar(s, "meanIntensity", m["preprocessing"]["meanIntensity"])
    s["sliceThicknesses"] = np.asarray(m["sliceThicknesses"], np.float64)
    _cx(s, "propagators", m["propagators"])
    _cx(s, "startSlices", m["startSlices"])
    _cx(s, "startProbe", m["startProbe"])
    _scalar(s, "cases", len(m["cases"]))
    for i, c in enumerate(m["cases"]):
        pre = f"case{i}_"
        for k in ("name", "slices", "fixProbeCenterOfMass", "constrainProbeAmplitude", "radius", "width", "fixProbe",
                  "purePhase", "identicalSlices"):
            _scalar(s, pre + k, c[k])
        s[pre + "thicknesses"] = np.asarray(c["thicknesses"], np.float64)
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    s["support"] = np.asarray(x["support"], np.bool_)
    extras = [c for c in x["cases"] if c["engine"] == "multislice"]
    _scalar(s, "extras", len(extras))
    for i, c in enumerate(extras):
        pre = f"extra{i}_"
        _scalar(s, pre + "name", c["name"])
        for k in ("fixProbeCenterOfMass", "fixProbeAperture", "fixProbe", "constrainProbeAmplitude", "radius", "width"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    return s


def options(fx):
    o = json.loads((fx / "options.json").read_text())
    s = {}
    a = o["objectAmplitude"]
    _cx(s, "startObject", a["startObject"])
    _scalar(s, "amplitudeCases", len(a["cases"]))
    for i, c in enumerate(a["cases"]):
        pre = f"amp{i}_"
        for k in ("name", "fixProbe", "purePhase", "step", "iterations", "maxAmplitude"):
            _scalar(s, pre + k, c[k])
        _cx(s, pre + "object", c["object"])
        _cx(s, pre + "probe", c["probe"])
        s[pre + "errors"] = np.asarray(c["errors"], np.float64)
    g = o["probes"]
    for k in ("rows", "columns", "rowSampling", "columnSampling", "wavelength", "cutoff", "rolloff"):
        _scalar(s, "probes_" + k, g[k])
    _scalar(s, "probeCases", len(g["cases"]))
    for i, c in enumerate(g["cases"]):
        pre = f"probe{i}_"
        for k in ("name", "defocus", "astigmatism", "astigmatismAngle", "sphericalAberration"):
            _scalar(s, pre + k, c[k])
        s[pre + "terms"] = np.asarray([[t["n"], t["m"], t["magnitude"], t["azimuth"]] for t in c["terms"]], np.float64).reshape(-1, 4)
        _cx(s, pre + "probe", c["probe"])
    _scalar(s, "appCases", len(o["appTranscription"]))
    for i, c in enumerate(o["appTranscription"]):
        pre = f"app{i}_"
        for k in ("name", "defocus", "c12a", "c12b"):
            _scalar(s, pre + k, c[k])
        s[pre + "terms"] = np.asarray([[t["radialOrder"], t["angularOrder"], 1.0 if t["sine"] else 0.0, t["coefficient"]]
                                       for t in c["terms"]], np.float64).reshape(-1, 4)
        _cx(s, pre + "probe", c["probe"])
    q = o["initialProbe"]
    for k in ("rows", "columns", "meanIntensity", "semiangle", "rolloff", "defocus", "astigmatism", "astigmatismAngle",
              "sphericalAberration", "samplingRow", "samplingColumn", "wavelength"):
        _scalar(s, "initial_" + k, q[k])
    s["initial_terms"] = np.asarray([[t["n"], t["m"], t["magnitude"], t["azimuth"]] for t in q["terms"]], np.float64).reshape(-1, 4)
    _cx(s, "initial_probe", q)
    return s


def preprocess(fx):
    q = json.loads((fx / "preprocess.json").read_text())
    s = {}
    for k in ("scanRows", "scanColumns", "detectorRows", "detectorColumns"):
        _scalar(s, k, q[k])
    for k in ("cube", "originRows", "originColumns"):
        s[k] = np.asarray(q[k], np.float64)
    for order, c in q["amplitudes"].items():
        s[f"order{order}_amplitudes"] = np.asarray(c["amplitudes"], np.float64)
        _scalar(s, f"order{order}_meanIntensity", c["meanIntensity"])
        _scalar(s, f"order{order}_clippedMeanIntensity", c["clippedMeanIntensity"])
    return s


def positions(fx):
    q = json.loads((fx / "positions.json").read_text())
    s = {}
    for k in ("rows", "columns", "objectRows", "objectColumns", "rowSampling", "columnSampling", "meanIntensity"):
        _scalar(s, k, q[k])
    for k in ("nominalPositions", "truthPositions", "amplitudes"):
        s[k] = np.asarray(q[k], np.float64)
    _cx(s, "startObject", q["startObject"])
    _cx(s, "startProbe", q["startProbe"])
    e = q["exact"]
    s["exact_amplitudes"] = np.asarray(e["amplitudes"], np.float64)
    _scalar(s, "exact_meanIntensity", e["meanIntensity"])
    _cx(s, "exact_object", e["object"])
    _cx(s, "exact_probe", e["probe"])
    s["exact_positions"] = np.asarray(e["positions"], np.float64)
    s["exact_errors"] = np.asarray(e["errors"], np.float64)
    names = []
    for c in q["cases"]:
        name = c["name"]
        names.append(name)
        st = c["settings"]
        # settings: stepSize, maxUpdateDistance (NaN = none), maxTotalDistance (NaN = none), constrainCenterOfMass
        s[f"case_{name}_settings"] = np.asarray([st["stepSize"], st.get("maxUpdateDistance", np.nan),
                                                 st.get("maxTotalDistance", np.nan),
                                                 1.0 if st.get("constrainCenterOfMass", False) else 0.0])
        _scalar(s, f"case_{name}_fixProbe", bool(c["fixProbe"]))
        _cx(s, f"case_{name}_object", c["object"])
        _cx(s, f"case_{name}_probe", c["probe"])
        s[f"case_{name}_errors"] = np.asarray(c["errors"], np.float64)
        s[f"case_{name}_positions"] = np.asarray(c["positions"], np.float64)
    s["cases"] = np.asarray(names)
    return s


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <CuboKit source tree>")
    root = Path(sys.argv[1])
    fx = root / "Tests/CuboPtychoTests/Fixtures"
    for name, fn in (("ptycho", ptycho), ("odd", odd), ("engines", engines), ("options", options),
                     ("preprocess", preprocess), ("positions", positions), ("mixed", mixed),
                     ("multislice", multislice)):
        arrays = fn(fx)
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, len(arrays), "arrays", (HERE / f"{name}.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main()
