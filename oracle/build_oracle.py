"""Builds the test oracle (TEST INFRASTRUCTURE ONLY; never linked by the product).

  oracle/_build/liboracle.so  -- the C restatement in oracle/oracle.c
  oracle/_ref/libref_util.so  -- the reference's own host-side operator tables
                                 (util/*.cpp from the reference checkout) behind
                                 the C shim oracle/ref_util/shim.cpp; built only
                                 when the reference sources are present.

The reference's OpenCL execution path itself is not buildable here (it needs
OpenCL headers and a platform, libtiff and Random123); only its self-contained
util/ sources are compiled, directly from where they lie, with g++.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: MAP_REFERENCE_DIR, else a `reference` directory beside
# this repository's root (absent on machines that only run the prebuilt files).
REF = os.environ.get("MAP_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
UTIL_SOURCES = ["DataType", "VariantType", "UnaryType", "BinaryType", "ReductionType", "NumDim", "MemOrder"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle():
    """Portable build (the checker of the tests; travels with the repository)."""
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if _stale(lib, [src]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", src, "-lm", "-o", lib])
    return lib


def _host_cpu_tag():
    import hashlib
    import platform
    info = platform.machine()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.strip() == "":
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:10]


def build_oracle_native():
    """-O3 -march=native build for timing the CPU baseline, compiled on the
    machine that runs it (the file name carries a digest of the host CPU model
    and flags, so a build made elsewhere is never loaded). Same semantics:
    -ffp-contract=off keeps every operation rounded once."""
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "liboracle_native_%s.so" % _host_cpu_tag())
    src = os.path.join(HERE, "oracle.c")
    if _stale(lib, [src]):
        _run(["gcc", "-O3", "-march=native", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", src,
              "-lm", "-o", lib])
    return lib


def build_ref_util():
    """Returns the path of libref_util.so, or None when the reference is absent."""
    util = os.path.join(REF, "util")
    out_dir = os.path.join(HERE, "_ref")
    lib = os.path.join(out_dir, "libref_util.so")
    if not os.path.isdir(util):
        return lib if os.path.exists(lib) else None
    os.makedirs(out_dir, exist_ok=True)
    srcs = [os.path.join(util, s + ".cpp") for s in UTIL_SOURCES]
    shim = os.path.join(HERE, "ref_util", "shim.cpp")
    compat = os.path.join(HERE, "ref_util", "compat.h")
    if _stale(lib, srcs + [shim, compat]):
        _run(["g++", "-std=c++11", "-O1", "-fPIC", "-shared", "-w", "-include", compat, "-I" + REF] + srcs + [shim, "-o", lib])
    return lib


if __name__ == "__main__":
    print(build_oracle())
    print(build_ref_util())
    sys.exit(0)
