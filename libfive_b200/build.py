"""Builds libfive_b200/lib/libfive.so (the C ABI + CUDA kernels for sm_100a).

Every .cpp under csrc/ is compiled with g++ and every .cu with nvcc for
sm_100a; objects go to libfive_b200/_build/ and the shared library to
libfive_b200/lib/.  Both host and device code are compiled without
floating-point contraction (-ffp-contract=off / -fmad=false) so that each
clause of a tape is evaluated as separately rounded IEEE operations.

Usage: python -m libfive_b200.build [--force]
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libfive.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I", os.path.join(ROOT, "include"), "-I", CSRC,
            "-I", os.path.join(CUDA_HOME, "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall",
            "-Wno-unused-function"]
NVCCFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-fmad=false",
                    "-Xcompiler", "-fPIC,-ffp-contract=off",
                    "--expt-relaxed-constexpr"]


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cpp") or name.endswith(".cu"):
            out.append(os.path.join(CSRC, name))
    return out


def _headers():
    return [os.path.join(CSRC, n) for n in os.listdir(CSRC)
            if n.endswith((".h", ".hpp", ".cuh"))] + [
        os.path.join(ROOT, "include", n)
        for n in os.listdir(os.path.join(ROOT, "include"))]


# Headers that kernels compiled at run time (csrc/jit.cpp) include; their
# text is built into the library.
JIT_HEADERS = ["opcode_ids.h", "scalar_minmax.h", "scalar_ops.h", "dev_interval.cuh",
               "dev_point.cuh"]


def _jit_headers_source():
    """Writes _build/jit_headers.cpp (the JIT headers as string literals)
    when a header is newer than it; returns its path."""
    out = os.path.join(BUILD, "jit_headers.cpp")
    srcs = [os.path.join(CSRC, h) for h in JIT_HEADERS]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(h) for h in srcs):
        return out
    delim = "lfbjit"
    parts = []
    for h in srcs:
        text = open(h).read()
        assert ")" + delim + '"' not in text
        parts.append('R"%s(%s)%s"' % (delim, text, delim))
    with open(out, "w") as f:
        f.write("// Generated by libfive_b200/build.py from csrc/: the headers that\n"
                "// kernels compiled at run time include.\n"
                "namespace lfb {\n"
                "extern const int kJitHeaderCount = %d;\n" % len(srcs) +
                "extern const char* const kJitHeaderNames[] = {%s};\n"
                % ", ".join('"%s"' % h for h in JIT_HEADERS) +
                "extern const char* const kJitHeaderSources[] = {\n%s};\n"
                % ",\n".join(parts) +
                "}  // namespace lfb\n")
    return out


def _compile(src, force, newest_header):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src),
                                             newest_header)):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCCFLAGS + INCLUDES + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXXFLAGS + INCLUDES + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(force=False, verbose=True):
    """Compiles (incrementally) and links the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in _headers())
    srcs = _sources() + [_jit_headers_source()]
    objs = []
    errors = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for obj, err in ex.map(lambda s: _compile(s, force, newest_header), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("\n".join(errors))
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + [
            "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
