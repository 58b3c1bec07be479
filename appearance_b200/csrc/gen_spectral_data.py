"""Writes spectral_data.h: measured data tables of the reference's spectral
tracer that this library uses as data.

The reference's CPU tracer (crates/appearance-path-tracer) makes every
metallic material (metallic > 0.9) a gold conductor, with the complex index of
refraction of gold as interleaved (wavelength nm, value) pairs in
radiometry/data_tables/materials.rs (AU_ETA, AU_K; pbrt-v4's measured data).
This script reads those two tables from a checkout of the reference and
writes them unchanged (the same decimal literals) as C arrays:

    python appearance_b200/csrc/gen_spectral_data.py <reference checkout>
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = "crates/appearance-path-tracer/src/radiometry/data_tables/materials.rs"


def table(src: str, name: str):
    m = re.search(r"pub const " + name + r": &\[f32\] = &\[(.*?)\];", src, re.S)
    if not m:
        raise SystemExit(f"{name} not found")
    vals = [v.strip() for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
    return vals[0::2], vals[1::2]


def main(ref_root: str):
    with open(os.path.join(ref_root, TABLE)) as f:
        src = f.read()
    lam_e, eta = table(src, "AU_ETA")
    lam_k, k = table(src, "AU_K")
    assert lam_e == lam_k, "the two gold tables sample the same wavelengths"

    def arr(name, macro, vals):
        rows = [", ".join(v + "f" for v in vals[i:i + 6]) for i in range(0, len(vals), 6)]
        return (f"#define {macro} \\\n    " + ", \\\n    ".join(rows) + "\n"
                f"constexpr float {name}[{len(vals)}] = {{{macro}}};\n")

    out = ["// Generated by gen_spectral_data.py from the reference's data tables",
           "// (radiometry/data_tables/materials.rs: AU_ETA, AU_K): the complex index of",
           "// refraction of gold, eta + i k, sampled at kAuSamples wavelengths (nm),",
           "// interpolated linearly in between (PiecewiseLinearSpectrum).  Data only;",
           "// the macros let device code define its own copies of the arrays.",
           "#pragma once", "", "namespace spec {", "",
           f"constexpr int kAuSamples = {len(lam_e)};",
           arr("kAuLambda", "SPEC_AU_LAMBDA", lam_e), arr("kAuEta", "SPEC_AU_ETA", eta),
           arr("kAuK", "SPEC_AU_K", k), "}  // namespace spec", ""]
    with open(os.path.join(HERE, "spectral_data.h"), "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
