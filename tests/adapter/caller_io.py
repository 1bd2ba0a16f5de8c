"""Input and output files of tests/adapter/sdl_caller.cc, and its build
(test infrastructure for tests/test_adapter.py and tests/test_gpu_adapter.py)."""
from __future__ import annotations

import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "tracklooper_b200")


def build(out_dir: str) -> str:
    """Compiles the caller against include/lst_sdl.hpp and links it to the
    in-tree library; returns the executable's path."""
    exe = os.path.join(out_dir, "sdl_caller")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "sdl_caller.cc"), "-o", exe, "-L", PKG, "-l:_lst_b200.so", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True)
    return exe


def write_input(path: str, inp) -> None:
    """One event: its Event-API inputs, then its LST::run inputs."""
    from tracklooper_b200.gen import PLS_FIELDS, SEED_FLOAT_FIELDS

    arrays = [(inp.x, np.float32), (inp.y, np.float32), (inp.z, np.float32), (inp.detId, np.uint32),
              (inp.idxInNtuple, np.uint32)]
    arrays += [(inp.pls[name], dt) for name, dt in PLS_FIELDS]
    s = inp.seeds
    arrays += [(s.see[name], np.float32) for name in SEED_FLOAT_FIELDS]
    arrays += [(s.see["see_q"], np.int32), (s.hit_offsets, np.uint32), (s.hit_idx, np.int32),
               (s.ph2_detId, np.uint32), (s.ph2_x, np.float32), (s.ph2_y, np.float32), (s.ph2_z, np.float32)]
    with open(path, "wb") as f:
        for a, dt in arrays:
            a = np.ascontiguousarray(a, dtype=dt)
            f.write(np.uint64(a.size).tobytes())
            f.write(a.tobytes())


def read_output(path: str) -> dict:
    names = [("counts", np.int64), ("tc_type", np.int16), ("tc_seed", np.int32), ("tc_hits", np.uint32),
             ("md_n", np.uint32), ("lst_hits", np.uint32), ("lst_len", np.uint32), ("lst_seedIdx", np.int32),
             ("lst_type", np.int16)]
    out = {}
    with open(path, "rb") as f:
        for name, dt in names:
            n = int(np.frombuffer(f.read(8), np.uint64)[0])
            out[name] = np.frombuffer(f.read(n * np.dtype(dt).itemsize), dt).copy()
    return out
