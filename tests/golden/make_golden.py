"""Regenerate the golden fixtures from the reference's own files, read as text.

The reference (motility-ddm) is JavaScript and cannot run where this project
is built, so its known-answer values are taken from its test sources and its
README and stored here as JSON:

  known_answers.json      constants asserted by test/t_kernels.mjs and
                          test/t_fft.mjs (J0, ln Gamma, window values, the
                          tolerances of every check)
  validation_matrix.json  the per-scenario outputs the reference publishes
                          for its 11-scenario matrix (README.md section 6)

Usage (needs a checkout of the reference's motility-ddm app):
    python tests/golden/make_golden.py <path to motility-ddm>
or set MOTILITY_DDM_REF to that path. Without either, it exits with a message.
"""
import json
import os
import re
import sys

REF = None  # the motility-ddm checkout, from the command line or MOTILITY_DDM_REF
HERE = os.path.dirname(os.path.abspath(__file__))


def _read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read().splitlines()


def _num_pairs(line):
    return [[float(a), float(b)] for a, b in re.findall(r"\[([-\d.e]+), ([-\d.e]+)\]", line)]


def known_answers():
    k = _read("test/t_kernels.mjs")
    j0_line = next(i for i, s in enumerate(k) if "for (const [x, ref] of" in s and "besselJ0" in k[i + 1])
    lg_line = next(i for i, s in enumerate(k) if "for (const [x, ref] of" in s and "lnGamma" in k[i + 1])
    j0 = _num_pairs(k[j0_line])
    # ln Gamma pairs mix literals and expressions (Math.log(24) ...): keep the
    # literal ones and restate the closed forms named in the same line.
    lg_src = k[lg_line]
    lg = [[1.0, 0.0]]
    if "Math.log(24)" in lg_src:
        lg.append([5.0, "ln(24)"])
    if "Math.log(Math.sqrt(Math.PI))" in lg_src:
        lg.append([0.5, "ln(sqrt(pi))"])
    m = re.search(r"\[10\.5, ([-\d.e]+)\]", lg_src)
    if m:
        lg.append([10.5, float(m.group(1))])
    f = _read("test/t_fft.mjs")
    w0 = next(s for s in f if "window w(0)" in s)
    return {
        "bessel_j0": {"source": f"motility-ddm/test/t_kernels.mjs:{j0_line + 1}",
                      "tol": 2e-8, "pairs": j0},
        "ln_gamma": {"source": f"motility-ddm/test/t_kernels.mjs:{lg_line + 1}",
                     "tol": 1e-12, "pairs": lg},
        "window": {"source": "motility-ddm/test/t_fft.mjs:72-77",
                   "w0": float(re.search(r"w\[0\] - ([\d.e-]+)\)", w0).group(1)),
                   "w_half": 1.0, "tol": 1e-12},
        "fft_vs_dft_rel": {"source": "motility-ddm/test/t_fft.mjs:24-40", "tol": 1e-12,
                           "round_trip": 1e-13},
        "spectrum2d_vs_dft": {"source": "motility-ddm/test/t_fft.mjs:43-69", "tol": 1e-12},
        "wk_vs_direct": {"source": "motility-ddm/test/t_fft.mjs:80-117", "D": 1e-11,
                         "C": 1e-11, "P": 1e-12, "D0": 1e-12},
        "phase_rotation": {"source": "motility-ddm/test/t_fft.mjs:120-137", "tol": 1e-12},
        "isf_quadrature": {"source": "motility-ddm/test/t_kernels.mjs:61-72", "tol": 2e-5},
        "isf2d_table": {"source": "motility-ddm/test/t_kernels.mjs:86-102", "tol": 2e-5},
        "nnls_kkt": {"source": "motility-ddm/test/t_kernels.mjs:108-134", "trials": 300},
        "varpro_recovery": {"source": "motility-ddm/test/t_kernels.mjs:137-163",
                            "vbar_rel": 1e-3, "Z_rel": 1e-2, "D_rel": 1e-2, "alpha_abs": 1e-3},
    }


def validation_matrix():
    lines = _read("README.md")
    start = next(i for i, s in enumerate(lines) if s.startswith("| Scenario | Truth | Verdict"))
    rows = {}
    for i in range(start + 2, len(lines)):
        s = lines[i]
        if not s.startswith("|"):
            break
        cells = [c.strip() for c in s.strip("|").split("|")]
        name, _truth, verdict, alpha, vbar, vmag = cells[:6]
        row = {"verdict": verdict, "source": f"motility-ddm/README.md:{i + 1}"}
        m = re.match(r"([\d.]+)", alpha)
        if m:
            row["alpha"] = float(m.group(1))
        m = re.match(r"([\d.]+)", vbar)
        if m:
            row["vbar"] = float(m.group(1))
        m = re.match(r"([\d.]+)(?: @ ([-\d]+)°)?", vmag)
        if m:
            row["V"] = float(m.group(1))
            if m.group(2):
                row["angle"] = float(m.group(2))
        rows[name] = row
    return rows


def main():
    if not os.path.isdir(REF):
        sys.exit("reference checkout not found")
    for name, data in (("known_answers.json", known_answers()),
                       ("validation_matrix.json", validation_matrix())):
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=1)
        print("wrote", name)


def _ref_path(argv):
    path = argv[1] if len(argv) > 1 else os.environ.get("MOTILITY_DDM_REF")
    if not path:
        sys.exit("make_golden.py: give the motility-ddm checkout as the first argument "
                 "or in MOTILITY_DDM_REF")
    if not os.path.isfile(os.path.join(path, "test", "t_kernels.mjs")):
        sys.exit(f"make_golden.py: {path} does not look like motility-ddm (no test/t_kernels.mjs)")
    return path


if __name__ == "__main__":
    REF = _ref_path(sys.argv)
    main()
