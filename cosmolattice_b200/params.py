"""Parameter files and run parameters, mirroring the reference's input handling.

* ``ParameterParser``: ``key = value`` text files with ``#`` comments plus ``key=value``
  command-line overrides (TempLat ParameterParser, used at source/cosmolattice.cpp:44).
* ``RunParameters``: the hot-path subset of include/CosmoInterface/runparameters.h:60-236 with
  the same keys, defaults and consistency checks (lSide = 2 pi / kIR = N dx, dt != 0, ...).
"""
from __future__ import annotations

import math
from typing import Dict, Iterable, List, Optional

from ._capi import EVOLVERS

RUN_PARAMETER_TOLERANCE = 1e-8  # runparameters.h:31


class RunParametersMissing(ValueError):
    """runparameters.h:20"""


class RunParametersInconsistent(ValueError):
    """runparameters.h:21"""


class NotAnEvolverType(ValueError):
    """evolvertype.h:15"""


def parse_evolver(value: str) -> int:
    """EvolverType from a name or its integer (evolvertype.h:39-82); LF, VV2-VV10 and PV2-PV10 exist
    here."""
    v = str(value).strip()
    if v in EVOLVERS:
        return EVOLVERS[v]
    if v.isdigit() and int(v) in EVOLVERS.values():
        return int(v)
    if v in ("RK2", "RK3_3", "RK3_4", "RK4_5") or (v.isdigit() and 7 <= int(v) <= 10):
        raise NotAnEvolverType(f"{v} is a reference evolver outside this library's hot path (LF, VV2-VV10, PV2-PV10).")
    raise NotAnEvolverType(f"{v} is not an evolver type, abort.")


def _almost_equal(a: float, b: float, eps: float = RUN_PARAMETER_TOLERANCE) -> bool:
    return abs(a - b) <= eps * max(1.0, abs(a), abs(b))


class ParameterParser:
    """``key = value`` parameters from a file and/or overrides, reference syntax."""

    def __init__(self, filename: Optional[str] = None, overrides: Optional[Iterable[str]] = None,
                 params: Optional[Dict[str, str]] = None):
        self.params: Dict[str, str] = {}
        if filename:
            with open(filename) as fh:
                self.read_text(fh.read())
        if params:
            self.params.update({k: str(v) for k, v in params.items()})
        for ov in overrides or ():
            if "=" not in ov:
                raise ValueError(f"override {ov!r} is not key=value")
            k, v = ov.split("=", 1)
            if k.strip() == "input":
                with open(v.strip()) as fh:
                    self.read_text(fh.read())
            else:
                self.params[k.strip()] = v.strip()

    @classmethod
    def from_argv(cls, argv: List[str]) -> "ParameterParser":
        """``input=<file> key=value ...`` as the reference executable takes them (README.md:35)."""
        return cls(overrides=argv)

    def read_text(self, text: str) -> None:
        for raw in text.splitlines():
            line = raw.split("#", 1)[0].strip()
            if not line or "=" not in line:
                continue
            k, v = line.split("=", 1)
            self.params[k.strip()] = v.strip()

    def has(self, key: str) -> bool:
        return key in self.params

    def get_str(self, key: str, default: Optional[str] = None) -> str:
        if key in self.params:
            return self.params[key]
        if default is None:
            raise RunParametersMissing(f"parameter {key!r} is required")
        return default

    def get_float(self, key: str, default: Optional[float] = None) -> float:
        if key in self.params:
            return float(self.params[key].split()[0])
        if default is None:
            raise RunParametersMissing(f"parameter {key!r} is required")
        return float(default)

    def get_floats(self, key: str, n: int, default: Optional[List[float]] = None) -> List[float]:
        if key in self.params:
            vals = [float(t) for t in self.params[key].split()]
            if len(vals) < n:
                raise RunParametersInconsistent(f"parameter {key!r} needs {n} values, got {len(vals)}")
            return vals[:n]
        if default is None:
            raise RunParametersMissing(f"parameter {key!r} is required")
        return list(default)

    def get_int(self, key: str, default: Optional[int] = None) -> int:
        if key in self.params:
            return int(float(self.params[key].split()[0]))
        if default is None:
            raise RunParametersMissing(f"parameter {key!r} is required")
        return int(default)

    def get_bool(self, key: str, default: Optional[bool] = None) -> bool:
        if key in self.params:
            v = self.params[key].strip().lower()
            if v in ("1", "true", "yes", "on"):
                return True
            if v in ("0", "false", "no", "off"):
                return False
            raise RunParametersInconsistent(f"parameter {key!r}={v!r} is not a boolean")
        if default is None:
            raise RunParametersMissing(f"parameter {key!r} is required")
        return bool(default)


class RunParameters:
    """Model-independent run parameters (runparameters.h:60-236), hot-path keys."""

    def __init__(self, par: ParameterParser):
        self.N = par.get_int("N")
        kIR = par.get_float("kIR", -1)
        lSide = par.get_float("lSide", -1)
        dx = par.get_float("dx", -1)
        self.dt = par.get_float("dt")
        self.expansion = par.get_bool("expansion", True)
        self.t0 = par.get_float("t0", 0.0)
        self.tMax = par.get_float("tMax", 10000 * self.dt)
        self.kCutoff = par.get_float("kCutOff", -1.0)
        self.tOutFreq = par.get_float("tOutputFreq", 10 * self.dt)
        self.tOutInfreq = par.get_float("tOutputInfreq", 100 * self.dt)
        self.tOutRareFreq = par.get_float("tOutputRareFreq", 1000 * self.dt)
        self.tOutVerb = par.get_float("tOutputVerb", 100 * self.dt)
        self.baseSeed = par.get_str("baseSeed", "0")
        self.outFn = par.get_str("outputfile", "./")
        self.fixedBackground = par.get_bool("fixedBackground", False) if self.expansion else False
        # fixed background (runparameters.h:90-94): equation of state and initial Hubble rate (GeV)
        self.omegaEoS = par.get_float("omegaEoS", 1.0 / 3.0) if self.fixedBackground else 1.0 / 3.0
        self.H0 = par.get_float("H0", 0.0) if self.fixedBackground else 0.0
        self.a0 = par.get_float("a0", 1.0)
        self.deltaKBin = par.get_float("deltaKBin", 1.0)
        self.nBinsSpectra = int(math.floor(math.sqrt(3.0) / 2.0 * self.N / self.deltaKBin))  # runparameters.h:98
        self.eType = parse_evolver(par.get_str("evolver", "LF"))
        self.appendMode = par.get_bool("appendToFiles", False)
        self.overwriteMode = par.get_bool("overwriteFiles", False)
        self.printHeaders = par.get_bool("print_headers", False)
        self.powerSpectrumType = par.get_int("PS_type", 1)
        self.powerSpectrumVersion = par.get_int("PS_version", 1)
        self.withGWs = par.get_bool("withGWs", False)
        self.doLFforGWs = par.get_bool("doLFforGWs", True)      # runparameters.h:121
        self.GWprojectorType = par.get_int("GWprojectorType", 2)  # runparameters.h:122-123

        # lSide = 2 pi / kIR = N dx (runparameters.h:155-186)
        hasK = not _almost_equal(kIR, -1)
        hasL = not _almost_equal(lSide, -1)
        hasD = not _almost_equal(dx, -1)
        if not (hasK or hasL or hasD):
            raise RunParametersMissing("You need to specify either kIR, lSide or dx, abort.")
        if not hasL:
            lSide = 2 * math.pi / kIR if hasK else dx * self.N
        if hasK and not _almost_equal(kIR, 2 * math.pi / lSide):
            raise RunParametersInconsistent(
                f"kIR = {kIR} and lSide = {lSide} are not consistent. If you think they should be, try removing one of the two.")
        if hasD and not _almost_equal(dx, lSide / self.N):
            raise RunParametersInconsistent(
                f"dx = {dx} and lSide = {lSide} (with N = {self.N}) are not consistent.")
        self.lSide = lSide
        self.kIR = 2 * math.pi / lSide
        self.dx = lSide / self.N

        if self.appendMode and self.overwriteMode:
            raise RunParametersInconsistent("'appendToFiles' and 'overwriteFiles' cannot both be true. Pick one.")
        if _almost_equal(self.dt, 0.0):
            raise RunParametersInconsistent("dt cannot be zero, abort.")
        if self.tMax < self.t0:
            raise RunParametersInconsistent("tMax must be >= t0, abort.")
        for name in ("tOutFreq", "tOutInfreq", "tOutRareFreq", "tOutVerb"):
            if getattr(self, name) < self.dt:
                raise RunParametersInconsistent(f"{name} must be >= dt, abort.")
        kUV = math.sqrt(3) * math.pi / self.dx
        if self.kCutoff < 0.0:
            self.kCutoff = 2 * kUV
        if self.powerSpectrumType not in (1, 2):
            raise RunParametersInconsistent(f"powerSpectrumType {self.powerSpectrumType} is not a valid powerSpectrumType.")
        if self.powerSpectrumVersion not in (1, 2, 3):
            raise RunParametersInconsistent(
                f"powerSpectrumVersion {self.powerSpectrumVersion} is not a valid powerSpectrumVersion.")
        if self.fixedBackground and _almost_equal(self.H0, 0.0):
            # FixedBackgroundExpansion ctor (fixedbackgroundexpansion.h:28-31), non-defect models
            raise RunParametersInconsistent(
                "For models that do not involve cosmic defects, you need to specify a non-zero H0 to run a simulation "
                "with fixed background. If you want to disable expansion, please set expansion = false in the input file.")
        if self.withGWs and not self.doLFforGWs:
            raise RunParametersInconsistent("GWs run as the reference's default leapfrog over the matter evolver "
                                            "(doLFforGWs = true) here.")
        if self.withGWs and self.GWprojectorType not in (1, 2, 3):
            raise RunParametersInconsistent(f"GWprojectorType {self.GWprojectorType} is not 1, 2 or 3.")
