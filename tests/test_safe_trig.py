"""Safe-trig source invariants of the variation library (CPU, no GPU).

The reference pins these in src/chaos-safetrig.gpu.test.ts by scanning
chaos.wgsl: named variations route cliff-prone trig arguments through
safe_sin / safe_cos / safe_tanh, and a forward scan flags raw trig in any
variation outside an audited allowlist.  Here the same checks scan the
generated-kernel sources (pyr3_b200/csrc/jit/vlib_*.cuh), whose wrappers are
ssin / scos / ssincos / stan (the argument through safe_arg) and stanh (the
argument clamped), and polar2 (ssincos)."""
import glob
import os
import re

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = "\n".join(open(f).read() for f in sorted(glob.glob(os.path.join(HERE, "..", "pyr3_b200", "csrc",
                                                                        "jit", "vlib_*.cuh"))))
# raw trig: a libm / intrinsic call not prefixed by a word character
RAW = re.compile(r"(?<![A-Za-z0-9_])(sinf|cosf|tanf|tanhf|sincosf|__sinf|__cosf|__tanf|ol_sincos|sin|cos|tan|tanh)\(")
SAFE_SINCOS = re.compile(r"(?<![A-Za-z0-9_])(ssin|scos|ssincos|stan|polar2)\(")


def _bodies(kind: str) -> dict:
    out = {}
    for m in re.finditer(r"\b" + kind + r"\((\w+)\)\s*\{", SRC):
        i, d = m.end(), 1
        while d:
            d += {"{": 1, "}": -1}.get(SRC[i], 0)
            i += 1
        out[m.group(1)] = re.sub(r"//[^\n]*", "", SRC[m.start():i])
    return out


VARS = _bodies("VAR")
DCS = _bodies("DCV")

# The reference's audited raw-trig allowlist (src/chaos-safetrig.gpu.test.ts,
# RAW_TRIG_OK: freshly atan2'd or bounded angles, the circular hash, the
# bsplit guard), without hypertile, hypertile2 and kaleidoscope, which route
# through the safe wrappers here; newton_color is the newton direct colour.
RAW_TRIG_OK = {"circus", "cardioid", "chrysanthemum", "bsplit", "circular", "circular2", "circleblur",
               "hypertile1", "idisc", "lace_js", "fourth", "cannabis_curve_wf", "e_collide", "e_mod",
               "b_mod", "waves4", "circlecrop", "billiard_sinai", "billiard_polygon", "quasicrystal",
               "penrose", "crackle", "hole"}
RAW_TRIG_OK_DC = {"newton"}


def test_safe_wrappers_guard_their_arguments():
    core = open(os.path.join(HERE, "..", "pyr3_b200", "csrc", "jit", "vlib_core.cuh")).read()
    assert re.search(r"VDEV float ssin\(float a\) \{ return sinf\(safe_arg\(a\)\); \}", core)
    assert re.search(r"VDEV float scos\(float a\) \{ return cosf\(safe_arg\(a\)\); \}", core)
    assert re.search(r"VDEV float stanh\(float a\) \{ return tanhf\(wclamp\(a, -20\.0f, 20\.0f\)\); \}", core)
    assert "ol_sincos(safe_arg(a))" in core


@pytest.mark.parametrize("name", ["waves", "tancos", "funnel", "clifford_js", "murl2", "phoenix_julia",
                                  "e_julia"])
def test_named_variations_use_safe_sin_cos(name):
    """#72 (waves), #235 (tancos, funnel), #262 audit (clifford_js, murl2,
    phoenix_julia, e_julia): safe sin/cos and no raw sin/cos."""
    b = VARS[name]
    assert SAFE_SINCOS.search(b), name
    assert not re.search(r"(?<![A-Za-z0-9_])(sinf|cosf|sincosf|__sinf|__cosf|ol_sincos|sin|cos)\(", b), name


@pytest.mark.parametrize("name", ["funnel", "tancos", "tractrix", "dc_cylinder"])
def test_unbounded_tanh_uses_safe_tanh(name):
    """#262: tanh of an unbounded coordinate goes through stanh (the
    dc_cylinder direct colour included)."""
    for b in ([VARS[name]] + ([DCS[name]] if name in DCS else [])):
        if "tanh" in b:
            assert "stanh(" in b and not re.search(r"(?<![A-Za-z0-9_])tanhf?\(", b), name
    assert "stanh(" in VARS[name] or "stanh(" in DCS.get(name, "")


def test_bsplit_guard_and_safe_cos():
    """bsplit keeps raw sin/cos of x + P[0] for its hide guard; the
    orthogonal cos(y + P[1]) goes through scos."""
    assert "scos(p.y + P[1])" in VARS["bsplit"]


def test_forward_scan_raw_trig_only_on_the_allowlist():
    """#306: every variation (and direct colour) with raw trig is on the
    audited allowlist, and no allowlisted name has become safe."""
    assert len(VARS) >= 300 and len(DCS) >= 10  # the scan ran over the catalog
    raw = {n for n, b in VARS.items() if RAW.search(b)}
    raw_dc = {n for n, b in DCS.items() if RAW.search(b)}
    assert raw - RAW_TRIG_OK == set(), sorted(raw - RAW_TRIG_OK)
    assert raw_dc - RAW_TRIG_OK_DC == set(), sorted(raw_dc)
    assert RAW_TRIG_OK - raw == set() and RAW_TRIG_OK_DC - raw_dc == set(), "stale allowlist entries"
