"""Writes t5dnn_reference.bin: the reference T5 classifier weights as
little-endian float32 in the order w0[38][32], b0[32], w2[32][32], b2[32],
w4[32], b4[1] (2337 values).

The weights live as C++ array initialisers in the reference header
SDL/NeuralNetworkWeights.h (T5DNN::wgtT_0, bias_0, wgtT_2, bias_2, wgtT_4,
bias_4).  The script lets g++ parse that header, so each decimal literal is
rounded to float exactly as the reference build rounds it, and dumps the
arrays.  Usage:

    python make_t5dnn_weights.py <reference checkout>/SDL [output.bin]
"""
import os
import subprocess
import sys
import tempfile

DUMP = r"""
#include <cstdio>
#define ALPAKA_STATIC_ACC_MEM_GLOBAL
#include "NeuralNetworkWeights.h"
int main(int argc, char** argv) {
  FILE* f = std::fopen(argv[1], "wb");
  if (!f) return 1;
  std::fwrite(T5DNN::wgtT_0, sizeof(float), 38 * 32, f);
  std::fwrite(T5DNN::bias_0, sizeof(float), 32, f);
  std::fwrite(T5DNN::wgtT_2, sizeof(float), 32 * 32, f);
  std::fwrite(T5DNN::bias_2, sizeof(float), 32, f);
  std::fwrite(T5DNN::wgtT_4, sizeof(float), 32, f);
  std::fwrite(T5DNN::bias_4, sizeof(float), 1, f);
  return std::fclose(f) == 0 ? 0 : 1;
}
"""


def main():
    sdl = sys.argv[1]
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                             "t5dnn_reference.bin")
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "alpaka"))
        open(os.path.join(tmp, "alpaka", "alpaka.hpp"), "w").close()
        src = os.path.join(tmp, "dump.cc")
        with open(src, "w") as f:
            f.write(DUMP)
        exe = os.path.join(tmp, "dump")
        subprocess.run(["g++", "-O0", "-I", tmp, "-I", sdl, src, "-o", exe], check=True)
        subprocess.run([exe, out], check=True)
    n = os.path.getsize(out) // 4
    if n != 2337:
        raise SystemExit(f"unexpected weight count {n}")
    print(f"wrote {out} ({n} floats)")


if __name__ == "__main__":
    main()
