"""Builds the checkers under oracle/ (test infrastructure only).

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


def build_all(reference_sdl: str | None = None) -> None:
    build_ref(reference_sdl or reference_sdl_dir())
