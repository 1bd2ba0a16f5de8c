"""The reference's C++ surface over the C ABI (include/lst_sdl.hpp): a
caller written against SDL::Event<SDL::Acc>, SDL::LST<SDL::Acc> and the
event-setup loaders (tests/adapter/sdl_caller.cc, in the style of bin/sdl.cc
and code/core/trkCore.cc) compiles unchanged and links to the library.
Running it needs a GPU (tests/test_gpu_adapter.py)."""
import os
import subprocess

import pytest

from tests.adapter import caller_io

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_api_caller_compiles_and_links(tmp_path):
    exe = caller_io.build(str(tmp_path))
    assert os.path.exists(exe)


def test_header_is_self_contained(tmp_path):
    src = tmp_path / "t.cc"
    src.write_text('#include "lst_sdl.hpp"\nint main() { SDL::QueueAcc q; (void)q; return 0; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                    os.path.join(ROOT, "include"), str(src)], check=True)


def test_caller_reports_a_bad_setup_without_aborting(tmp_path):
    """Without a GPU (or with a wrong LST_BASE) the caller ends with the
    library's error message, not a crash: the C ABI's status codes become
    exceptions in the adapter."""
    exe = caller_io.build(str(tmp_path))
    from tracklooper_b200 import gen

    inp = gen.generate_event(1, 0)
    path = tmp_path / "in.bin"
    caller_io.write_input(str(path), inp)
    env = dict(os.environ, LST_BASE=str(tmp_path / "nowhere"))
    r = subprocess.run([exe, str(path), str(tmp_path / "out.bin")], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1
    assert "sdl_caller:" in r.stderr and "sensor_centroids.bin" in r.stderr
