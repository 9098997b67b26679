"""Build recipe for the oracle (test infrastructure only).

* oracle/liboracle.so      -- the plain-C restatement (oracle/oracle.c);
* oracle/_ref/libpyr3_ref.so -- the reference's own WGSL shaders
  (src/shaders/{noise_perlin,chaos,density,visualize_u32,visualize_f32}.wgsl,
  read where they lie under the reference checkout) translated to C++ by
  oracle/wgsl2cpp.py and compiled with oracle/ref_glue.cpp;
* oracle/_ref/libpyr3_ref64.so -- the same chaos shader with every f32
  evaluated as a double (oracle/ref64_glue.cpp): the FP64 evaluation of the
  variations.

The reference checkout exists only in the build container; on a machine
without it the prebuilt oracle/_ref/libpyr3_ref.so (which travels with the
working tree) is used as is.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("PYR3_REFERENCE", "/root/reference")
REF_SHADERS = os.path.join(REF_ROOT, "src", "shaders")

CFLAGS = ["-O2", "-fPIC", "-shared", "-fwrapv", "-ffp-contract=off", "-fno-fast-math"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle() -> str:
    out = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        _run(["gcc", "-std=c11", *CFLAGS, src, "-o", out, "-lm"])
    return out


def build_reference() -> str | None:
    """Translate + compile the reference shaders; None if the reference
    sources are absent and no prebuilt library exists."""
    ref_dir = os.path.join(HERE, "_ref")
    out = os.path.join(ref_dir, "libpyr3_ref.so")
    if not os.path.isdir(REF_SHADERS):
        return out if os.path.exists(out) else None
    os.makedirs(ref_dir, exist_ok=True)
    sys.path.insert(0, HERE)
    import wgsl2cpp  # noqa: E402

    units = {
        "chaos": ["noise_perlin.wgsl", "chaos.wgsl"],
        "density": ["density.wgsl"],
        "visualize_u32": ["visualize_u32.wgsl"],
        "visualize_f32": ["visualize_f32.wgsl"],
    }
    deps = [os.path.join(HERE, f) for f in ("wgsl2cpp.py", "wgsl_rt.hpp", "ref_glue.cpp")]
    for files in units.values():
        deps += [os.path.join(REF_SHADERS, f) for f in files]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    for ns, files in units.items():
        srcs = [open(os.path.join(REF_SHADERS, f)).read() for f in files]
        code = wgsl2cpp.translate(srcs, ns, skip_fns=("vs",))
        with open(os.path.join(ref_dir, f"{ns}.cpp"), "w") as fh:
            fh.write(code + "\n")
    glue = os.path.join(HERE, "ref_glue.cpp")
    # The glue #includes the translated units relative to oracle/_ref/.
    shim = os.path.join(ref_dir, "ref_glue_tu.cpp")
    with open(shim, "w") as fh:
        fh.write(f'#include "{glue}"\n')
    _run(["g++", "-std=c++17", *CFLAGS, "-I", ref_dir, shim, "-o", out, "-lpthread"])
    return out


def build_reference_f64() -> str | None:
    """The reference's chaos shader translated with every f32 evaluated as
    a double (oracle/_ref/libpyr3_ref64.so): the FP64 evaluation the
    variations' f32 error is stated against.  None if the reference sources
    are absent and no prebuilt library exists."""
    ref_dir = os.path.join(HERE, "_ref")
    out = os.path.join(ref_dir, "libpyr3_ref64.so")
    if not os.path.isdir(REF_SHADERS):
        return out if os.path.exists(out) else None
    os.makedirs(ref_dir, exist_ok=True)
    sys.path.insert(0, HERE)
    import wgsl2cpp  # noqa: E402

    files = ["noise_perlin.wgsl", "chaos.wgsl"]
    deps = [os.path.join(HERE, f) for f in ("wgsl2cpp.py", "wgsl_rt.hpp", "ref64_glue.cpp")]
    deps += [os.path.join(REF_SHADERS, f) for f in files]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    srcs = [open(os.path.join(REF_SHADERS, f)).read() for f in files]
    code = wgsl2cpp.translate(srcs, "chaos64", skip_fns=("vs",), f32_type="double")
    with open(os.path.join(ref_dir, "chaos64.cpp"), "w") as fh:
        fh.write(code + "\n")
    shim = os.path.join(ref_dir, "ref64_glue_tu.cpp")
    with open(shim, "w") as fh:
        fh.write(f'#include "{os.path.join(HERE, "ref64_glue.cpp")}"\n')
    _run(["g++", "-std=c++17", *CFLAGS, "-I", ref_dir, shim, "-o", out])
    return out


def build_all() -> None:
    build_oracle()
    build_reference()
    build_reference_f64()


if __name__ == "__main__":
    build_all()
    print("oracle built")
