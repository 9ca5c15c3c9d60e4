"""Extract named definitions from the reference's CUDA/C++ sources into
include files under oracle/_ref/ (test infrastructure: nothing here is
shipped, and the extracted text stays out of the repository).

The reference cannot be built as a whole here (Eigen, CGAL, OpenVDB and a
GPU are missing), but some of its arithmetic is self-contained device code:
the Heaviside projection and penalty functions, the spline basis recursion,
the knot series, and the element kernels of the density map and the
sensitivity filter.  This script copies exactly those definitions, unmodified,
from the files where they lie; ref_golden.cpp compiles them on the host with
a shim for the CUDA keywords, and tests/golden/make_golden.py runs them to
write the golden fixtures the oracle is pinned against.

Each spec names a file, a regular expression matching the first line of the
definition, a mode, and optionally an anchor: a regular expression whose
first match starts the search (for a lambda whose text repeats in other
functions).  Modes:
  def   the definition from its first line (and a 'template<...>' line just
        above it) through its matching closing brace (and a ';' after it)
  body  only the brace-enclosed body of the matched function
  expr  from the match itself (not the line start) through the matching
        closing brace and its ';' (a lambda assigned to a variable)
"""
import os
import re
import sys

# (output include, source file relative to the reference root, regex, mode)
SPECS = [
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float Heaviside\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float Dirac\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float h\(float x", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float dh\(float x", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float inner_\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float dinner_\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float overhang\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float doverhang\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float normal_distri\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ float dnormal_distri\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisX\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisY\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisZ\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisDeriX\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisDeriY\(", "def"),
    ("grid_funcs.inc", "grid/Grid.cu", r"__device__ void SplineBasisDeriZ\(", "def"),
    ("grid_kernels.inc", "grid/Grid.cu", r"__global__ void coeff2density_kernel\(", "def"),
    ("grid_kernels.inc", "grid/Grid.cu", r"__global__ void filterSensitivity_kernel\(", "def"),
    ("calc_node.inc", "grid/Grid.cu", r"auto calc_node = \[=\] __device__\(int id\)", "expr"),
    ("filter_weight.inc", "grid/Grid.cu", r"auto fr = \[=\] __device__\(float r\)", "expr"),
    ("knots_body.inc", "grid/Grid.cpp", r"void grid::Grid::set_spline_knot_series\(void\)", "body"),
    ("opt_kernels.inc", "optimization/optimization.cu", r"__global__ void computeProjectionSensitivity_kernel\(", "def"),
    ("opt_kernels.inc", "optimization/optimization.cu", r"__global__ void computeProjection_kernel\(", "def"),
    ("lib_bits.inc", "culib/lib.cuh", r"__device__ bool read_gbit\(T word, int id\)", "def"),
    ("lib_bits.inc", "culib/lib.cuh", r"__device__ T clamp\(T value, T low, T upp\)", "def"),
    ("lib_bits.inc", "culib/lib.cuh", r"struct gBitSAT \{", "def"),
    # surface-point self-support (deal_surface_points, optimization/optimization.cpp:1185-1221)
    ("surf_funcs.inc", "grid/Grid.cu", r"__device__ float oh\(float x", "def"),
    ("surf_funcs.inc", "grid/Grid.cu", r"__device__ float doh\(float x", "def"),
    ("surf_funcs.inc", "grid/Grid.cu", r"__device__ float norm\(float v\[3\]\)", "def"),
    ("surf_funcs.inc", "grid/Grid.cu", r"__device__ float dot\(float v1\[3\]", "def"),
    ("surf_funcs.inc", "grid/Grid.cpp", r"std::vector<int> generateEquidistantIntegers\(int range", "def"),
    ("surf_mc.inc", "grid/Grid.cu", r"auto calc_node = \[=\] __device__\(int id\)", "expr",
     r"void Grid::compute_background_mcPoints_value\("),
    ("surf_normal.inc", "grid/Grid.cu", r"auto calc_normal = \[=\] __device__\(int node_id\)", "expr",
     r"void grid::Grid::compute_spline_surface_point_normal\(void\)"),
    ("surf_dir.inc", "grid/Grid.cu", r"auto calc_node = \[=\] __device__\(int node_id\)", "expr",
     r"float grid::Grid::correct_spline_surface_point_normal_direction\(float beta\)"),
    ("surf_flag.inc", "grid/Grid.cu", r"auto calc_node = \[=\] __device__\(int node_id\)", "expr",
     r"void grid::Grid::compute_selfsupp_flag_actual\(void\)"),
    ("surf_ss.inc", "grid/Grid.cu", r"auto calc_node = \[=\] __device__\(int node_id\)", "expr",
     r"void grid::Grid::compute_spline_selfsupp_constraint\(void\)"),
    ("surf_dss.inc", "grid/Grid.cu", r"auto calc_node_value = \[=\] __device__\(int node_id\)", "expr",
     r"void grid::Grid::compute_spline_selfsupp_constraint_dcoeff\(void\)"),
]


def _match_brace(text, start):
    """Index one past the brace that closes the first '{' at or after start,
    skipping comments, string and character literals."""
    i, depth, n = start, 0, len(text)
    opened = False
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
            continue
        if text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
            continue
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if c == "{":
            depth += 1
            opened = True
        elif c == "}":
            depth -= 1
            if opened and depth == 0:
                return i + 1
        i += 1
    raise ValueError("unbalanced braces")


def extract(text, pattern, mode, anchor=None):
    pos = 0
    if anchor:
        a = re.search(anchor, text)
        if not a:
            raise ValueError(f"anchor not found: {anchor}")
        pos = a.end()
    m = re.compile(pattern).search(text, pos)
    if not m:
        raise ValueError(f"pattern not found: {pattern}")
    if mode == "expr":
        begin = m.start()
    else:
        begin = text.rfind("\n", 0, m.start()) + 1
        # a template header on the line above belongs to the definition
        prev = text.rfind("\n", 0, begin - 1) + 1
        if mode == "def" and text[prev:begin].lstrip().startswith("template"):
            begin = prev
    end = _match_brace(text, m.start())
    if mode == "body":
        begin = text.find("{", m.start())
    rest = text[end:end + 8]
    if rest.lstrip().startswith(";"):
        end = text.find(";", end) + 1
    line = text.count("\n", 0, begin) + 1
    return line, text[begin:end]


def main(ref_root, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    chunks = {}
    for spec in SPECS:
        out, src, pattern, mode = spec[:4]
        anchor = spec[4] if len(spec) > 4 else None
        path = os.path.join(ref_root, src)
        with open(path, encoding="utf-8", errors="replace") as f:
            text = f.read()
        line, code = extract(text, pattern, mode, anchor)
        chunks.setdefault(out, []).append(f"// {src}:{line}\n#line {line} \"{src}\"\n{code}\n")
    for out, parts in chunks.items():
        with open(os.path.join(out_dir, out), "w") as f:
            f.write("".join(parts))
    print(f"extracted {len(SPECS)} definitions into {len(chunks)} files under {out_dir}")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
