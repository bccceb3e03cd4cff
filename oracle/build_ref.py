"""Build oracle/_ref/libcmgref.so from the reference's own sources (test infrastructure).

Recipe: the reference headers are used where they lie (-I into the reference
tree); the few function definitions that live in .cu files whose other
contents need libraries absent here (Eigen, TBB, polyscope) are cut out of
those files verbatim into a temporary directory at build time, next to a
symlink that gives the fmt headers bundled with spdlog the include path
<fmt/...>.  Only the compiled .so lands in oracle/_ref/ (git-ignored); no
reference source is written into the repository.

Usage: python oracle/build_ref.py [reference_root]
Exits 0 without building when the reference tree is absent and the library
is already built (a machine that only runs tests).
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libcmgref.so")
REF_DEFAULT = "/root/reference"

# (file, signature regex, namespace to wrap the definition in)
CUTCELL = [
    ("cirrus_cutcell/MeshCutCell.cu", r"__hostdev__\s+int\s+CellCornerSDFInsideCount\s*\(", None),
    ("cirrus_cutcell/MeshCutCell.cu", r"__hostdev__\s+float\s+FracInside\s*\(", None),
    ("cirrus_cutcell/MeshCutCell.cu", r"__hostdev__\s+float\s+FaceFluidRatio\s*\(\s*float", None),
]
SOLVERTESTS = [
    ("tests/SolverTests.cu", r"__hostdev__\s+int\s+SolverTestsLevelTarget\s*\(", "SolverTests"),
]
# the header struct that HADeviceGrid::dumpBinaryBlob writes (a local struct there)
HAGR = [
    ("src/HAGrid.h", r"struct\s+Header\s*\{", "ref_hagr"),
]


def fmt_include_dir():
    import sysconfig

    site = sysconfig.get_paths()["purelib"]
    cand = os.path.join(site, "flashinfer", "data", "spdlog", "include", "spdlog", "fmt", "bundled")
    return cand if os.path.isfile(os.path.join(cand, "core.h")) else None


def cut_definition(text, sig_re):
    """Return the text of the function whose signature matches sig_re, through its closing brace."""
    m = re.search(sig_re, text)
    if not m:
        raise RuntimeError(f"definition not found: {sig_re}")
    i = text.index("{", m.start())
    depth = 0
    for j in range(i, len(text)):
        c = text[j]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                line = text.count("\n", 0, m.start()) + 1
                return line, text[m.start(): j + 1]
    raise RuntimeError(f"unbalanced braces after {sig_re}")


def write_extract(ref, items, path):
    parts = []
    for rel, sig, ns in items:
        with open(os.path.join(ref, rel)) as f:
            text = f.read()
        line, body = cut_definition(text, sig)
        if body.startswith("struct"):
            body += ";"
        src = f'#line {line} "{os.path.join(ref, rel)}"\n{body}\n'
        if ns:
            src = f"namespace {ns} {{\n{src}}}\n"
        parts.append(src)
    with open(path, "w") as f:
        f.write("".join(parts))


def build(ref=REF_DEFAULT):
    if not os.path.isdir(ref):
        if os.path.exists(OUT):
            return OUT
        raise FileNotFoundError(f"reference tree {ref} absent and {OUT} not built")
    fmt = fmt_include_dir()
    if fmt is None:
        raise FileNotFoundError("bundled fmt headers not found")
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="cmgref_")
    try:
        os.symlink(fmt, os.path.join(tmp, "fmt"))
        write_extract(ref, CUTCELL, os.path.join(tmp, "ref_cutcell_extract.inc"))
        write_extract(ref, SOLVERTESTS, os.path.join(tmp, "ref_solvertests_extract.inc"))
        write_extract(ref, HAGR, os.path.join(tmp, "ref_hagr_extract.inc"))
        cmd = [
            "nvcc", "-std=c++17", "-O2", "--expt-extended-lambda", "--expt-relaxed-constexpr",
            "-gencode", "arch=compute_100a,code=sm_100a",
            "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
            "-include", "cfloat", "-DFMT_HEADER_ONLY",
            "-I", tmp,
            "-I", os.path.join(ref, "src"), "-I", os.path.join(ref, "ext"), "-I", os.path.join(ref, "common"),
            "-I", os.path.join(ref, "tests"), "-I", os.path.join(ref, "cirrus_cutcell"),
            os.path.join(HERE, "ref_harness.cu"), "-o", OUT,
        ]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("building oracle/_ref/libcmgref.so failed")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else REF_DEFAULT))
