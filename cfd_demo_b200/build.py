"""Build recipe of the native library ``libcfd_b200.so`` (sm_100a).

    python -m cfd_demo_b200.build          # or __graft_entry__.build()

Steps: (1) print the degree-4 reference-triangle tables as compile-time
constants into ``csrc/tables.cuh``; (2) compile the objects with nvcc for
``sm_100a`` in parallel — ``kernels.cu`` (limiter, adjoint, small kernels and
the C ABI) and ``stage_inst.cu`` once per precision x mode of the fused stage
kernels and ``batch_inst.cu`` once per precision x flux of the persistent
batch kernel — into ``_build/``, each rebuilt only when its inputs change; (3) link
them into ``cfd_demo_b200/libcfd_b200.so`` (in-tree, so it travels with the
repository snapshot). No CUDA device is needed to build.
"""

from __future__ import annotations

import hashlib
import os
from concurrent.futures import ThreadPoolExecutor
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libcfd_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
]
# (object name, source, extra defines)
OBJECTS = [("kernels", "kernels.cu", []), ("setup", "setup.cu", [])] + [
    (f"stage_{prec}_{mode}", "stage_inst.cu", [f"-DCFD_STAGE_PREC={p}", f"-DCFD_STAGE_MODE={m}"])
    for p, prec in enumerate(("f64", "f32")) for m, mode in enumerate(("rhs", "limited", "unlimited"))
] + [
    (f"batch_{prec}_{flux}", "batch_inst.cu", [f"-DCFD_BATCH_PREC={p}", f"-DCFD_BATCH_FLUX={f}"])
    for p, prec in enumerate(("f64", "f32")) for f, flux in enumerate(("rusanov", "roe", "hllc"))
]


def _fmt(v: float) -> str:
    return repr(float(v))


def _array(name: str, a: np.ndarray, ctype: str = "double") -> str:
    a = np.asarray(a)
    dims = "".join(f"[{d}]" for d in a.shape)
    if ctype == "int":
        body = ", ".join(str(int(v)) for v in a.ravel())
    elif ctype == "float":
        body = ", ".join(repr(float(np.float32(v))) + "f" for v in a.ravel())
    else:
        body = ", ".join(_fmt(v) for v in a.ravel())
    return f"__device__ constexpr {ctype} {name}{dims} = {{{body}}};\n"


def _packed(face_nodes: np.ndarray) -> int:
    """Face-node table packed 4 bits per entry, entry (f, k) at bit 4 (5 f + k)."""
    return sum(int(n) << (4 * (f * face_nodes.shape[1] + k)) for f, row in enumerate(face_nodes) for k, n in enumerate(row))


def generate_tables() -> str:
    from .reference_element import build_reference_triangle

    ref = build_reference_triangle(4)
    w = ref.cell_weights
    text = [
        "// tables.cuh — GENERATED by cfd_demo_b200/build.py from reference_element.py. Do not edit.\n",
        "// Degree-4 nodal triangle: Np = 15, 3 faces x 5 GLL nodes (CFD-demo\n",
        "// src/cfd_demo/reference_element.py:264-316 builds the same tables).\n",
        "#pragma once\nnamespace cfd { namespace tab {\n",
        _array("DR", ref.dr), _array("DS", ref.ds), _array("LIFT", ref.lift),
        _array("FACE_NODES", ref.face_nodes, "int"),
        f"constexpr unsigned long long FACE_NODES_PACKED = {_packed(ref.face_nodes)}ull;\n",
        _array("CELL_W", w), _array("AVG_W", w / w.sum()),
        _array("FACE_W", ref.face_weights[0]),
        _array("MID_NODES", ref.face_midpoint_nodes, "int"),
        _array("P1MID", ref.p1_midpoint), _array("LINBASIS", ref.linear_midpoint_basis),
        "}}  // namespace cfd::tab\n",
        "namespace cfd { namespace ctab {  // the same tables in the constant bank (warp-uniform runtime index)\n",
        _array("DR", ref.dr).replace("__device__ constexpr", "static __constant__"),
        _array("DS", ref.ds).replace("__device__ constexpr", "static __constant__"),
        _array("LIFT", ref.lift).replace("__device__ constexpr", "static __constant__"),
        _array("DR32", ref.dr, "float").replace("__device__ constexpr", "static __constant__"),
        _array("DS32", ref.ds, "float").replace("__device__ constexpr", "static __constant__"),
        _array("LIFT32", ref.lift, "float").replace("__device__ constexpr", "static __constant__"),
        _array("AVG_W", w / w.sum()).replace("__device__ constexpr", "static __constant__"),
        _array("FACE_NODES", ref.face_nodes, "int").replace("__device__ constexpr", "static __constant__"),
        _array("FACE_W", ref.face_weights[0]).replace("__device__ constexpr", "static __constant__"),
        "}}  // namespace cfd::ctab\n",
    ]
    assert np.allclose(ref.face_weights, ref.face_weights[0][None]), "faces share one GLL rule"
    return "".join(text)


def _digest(paths, extra=()) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join([*NVCC_FLAGS, *extra]).encode())
    return h.hexdigest()


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _compile(name: str, source: str, defines: list[str], headers: list[str], force: bool) -> tuple[str, bool, str]:
    """Compile one object unless its digest (sources + flags) is unchanged."""
    obj = os.path.join(BUILD_DIR, name + ".o")
    stamp = obj + ".sha256"
    digest = _digest([os.path.join(CSRC, source), *headers], defines)
    if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == digest:
        return obj, False, ""
    cmd = [_nvcc(), *NVCC_FLAGS, *defines, f"-I{INCLUDE}", f"-I{CSRC}", "-c", os.path.join(CSRC, source),
           "-o", obj + ".tmp"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed ({proc.returncode}): {' '.join(cmd)}")
    os.replace(obj + ".tmp", obj)
    with open(stamp, "w") as f:
        f.write(digest)
    with open(obj + ".ptxas.txt", "w") as f:
        f.write(proc.stderr)
    return obj, True, proc.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Generate the tables, compile the changed objects in parallel and link
    the library if any object changed."""
    tables = os.path.join(CSRC, "tables.cuh")
    text = generate_tables()
    if not os.path.exists(tables) or open(tables).read() != text:
        with open(tables, "w") as f:
            f.write(text)
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc")))
    headers.append(os.path.join(INCLUDE, "cfd_b200.h"))
    with ThreadPoolExecutor(max_workers=min(len(OBJECTS), os.cpu_count() or 1)) as pool:
        results = list(pool.map(lambda o: _compile(*o, headers, force), OBJECTS))
    objs = [r[0] for r in results]
    stamp = LIB + ".sha256"
    digest = _digest(objs)
    if any(r[1] for r in results) or force or not os.path.exists(LIB) or not os.path.exists(stamp) \
            or open(stamp).read() != digest:
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB + ".tmp"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            sys.stderr.write(proc.stdout + proc.stderr)
            raise RuntimeError(f"nvcc link failed ({proc.returncode}): {' '.join(cmd)}")
        os.replace(LIB + ".tmp", LIB)
        with open(stamp, "w") as f:
            f.write(digest)
    with open(os.path.join(HERE, "ptxas_report.txt"), "w") as f:
        for name, _, _ in OBJECTS:
            with open(os.path.join(BUILD_DIR, name + ".o.ptxas.txt")) as g:
                f.write(g.read())
    if verbose:
        for r in results:
            sys.stdout.write(r[2])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
