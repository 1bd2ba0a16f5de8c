"""Builds the checkers under oracle/ (test infrastructure only).

* oracle/_ref/liblsttrace.so: the cut-flip tracer and FP64 re-evaluation
  (oracle/trace/lst_trace.cc over the product's cut headers and its
  event-setup loader), built from this repository's sources alone.
* oracle/_ref/liblstref_*.so: the reference CPU backend compiled from the
  reference sources (SDL/*.cc) against the serial Alpaka shim, by
  oracle/ref/Makefile.  Needs the reference checkout, found through the
  LST_REFERENCE_SDL environment variable (the checkout's SDL/ directory) or,
  without it, at the reference checkout's location in the build container;
  where neither exists the prebuilt libraries are used as they are.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REFERENCE_SDL = "/root/reference/SDL"


def reference_sdl_dir() -> str | None:
    """The reference's SDL/ source directory, or None where it is absent."""
    d = os.environ.get("LST_REFERENCE_SDL") or DEFAULT_REFERENCE_SDL
    return d if os.path.isdir(d) else None


def build_ref(reference_sdl: str | None) -> None:
    if not reference_sdl:
        return
    jobs = str(max(1, min(8, os.cpu_count() or 1)))
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF_SDL={reference_sdl}", "-j", jobs],
                   check=True)


ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "tracklooper_b200", "csrc")
TRACER = os.path.join(HERE, "_ref", "liblsttrace.so")


def build_tracer(force: bool = False) -> str:
    """Compiles the tracer without optimisation (every comparison stays an
    out-of-line call whose return address names its source line)."""
    srcs = [os.path.join(HERE, "trace", "lst_trace.cc"), os.path.join(CSRC, "es.cc")]
    deps = srcs + [os.path.join(HERE, "trace", "tfloat.h")] + [
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    if not force and os.path.exists(TRACER) and all(os.path.getmtime(d) <= os.path.getmtime(TRACER) for d in deps):
        return TRACER
    os.makedirs(os.path.dirname(TRACER), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O0", "-g", "-fno-omit-frame-pointer", "-fPIC", "-shared", "-I", CSRC,
           "-I", os.path.join(HERE, "trace"), "-o", TRACER + ".tmp"] + srcs + ["-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(TRACER + ".tmp", TRACER)
    return TRACER


def build_all(reference_sdl: str | None = None) -> None:
    build_tracer()
    build_ref(reference_sdl or reference_sdl_dir())
