"""Builds the reference's own runtime -- its DAG, online simplifier, fusion
compiler and OpenCL kernel generators -- from the reference checkout's sources,
for the CPU, linked against the stand-in OpenCL / libtiff entry points of
stubs.cpp, plus driver.cpp: oracle/_ref/ref_codegen (TEST INFRASTRUCTURE ONLY;
never linked by the product).

Compiles the source list of the reference's Makefile (S_* variables) directly
from where the files lie, with g++ and this directory's forced-include
compatibility header; nothing is copied. Outputs go to oracle/_ref/ only.
The reference checkout: MAP_REFERENCE_DIR, else `reference` beside this
repository's root. Returns None when it is absent.
"""
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
REF = os.environ.get("MAP_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(ORACLE)), "reference")
OUT = os.path.join(ORACLE, "_ref")
OBJ = os.path.join(OUT, "codegen_obj")
EXE = os.path.join(OUT, "ref_codegen")


def makefile_sources(ref):
    text = open(os.path.join(ref, "Makefile")).read().replace("\r", "")
    srcs = []
    for m in re.finditer(r"^S_[A-Z]+\s*=\s*\$\(addprefix\s+([^,]+),\s*([^)]*)\)", text, re.M):
        d = m.group(1).strip()
        srcs += [d + f for f in m.group(2).split()]
    return srcs


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout[-4000:]))


def build():
    if not os.path.isfile(os.path.join(REF, "Makefile")):
        return None
    os.makedirs(OBJ, exist_ok=True)
    # -O0 -fno-unreachable-traps: some reference functions declared to return a
    # value end without a return statement (file/File.cpp IFile::setDataStats);
    # current GCC turns that into a trap (or, optimising, into a fall-through
    # into the next function), so they are compiled the way the compilers of the
    # reference's time treated them: returning whatever the register holds.
    flags = ["-std=c++11", "-O0", "-fno-unreachable-traps", "-w", "-fpic", "-pthread", "-include",
             os.path.join(HERE, "compat.h"),
             "-I" + os.path.join(HERE, "stub")]
    mine = [os.path.join(HERE, "stubs.cpp"), os.path.join(HERE, "driver.cpp")]
    deps = [os.path.join(HERE, "compat.h"), os.path.join(HERE, "stub", "CL", "cl.h"), os.path.join(HERE, "stub", "tiffio.h")]
    newest_dep = max(os.path.getmtime(d) for d in deps + [os.path.abspath(__file__)])
    jobs, objs = [], []
    for rel in makefile_sources(REF):
        src = os.path.join(REF, rel)
        obj = os.path.join(OBJ, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_dep):
            jobs.append(["g++"] + flags + ["-c", src, "-o", obj])
    for src in mine:
        obj = os.path.join(OBJ, "own_" + os.path.basename(src) + ".o")
        objs.append(obj)
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_dep):
            jobs.append(["g++"] + flags + ["-I" + REF, "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(_run, jobs))
    if jobs or not os.path.exists(EXE):
        _run(["g++", "-pthread", "-o", EXE] + objs)
    return EXE


if __name__ == "__main__":
    print(build())
    sys.exit(0)
