"""Regenerate the fixtures of tests/golden/ from the reference's own files:
fft_rect_double.npz from its FFT golden vectors, hre_lomacte3.dat /
hre_lomacte.dat, verbatim copies of the run-parameter files of the two
lomacte codes (trunk/lomacte3/hre.dat, trunk/lomacte/hre.dat) that
tests/test_files.py parses as initcr does, and mesh_*.txt, verbatim copies
of three of the y meshes the reference's initial-condition generator reads
(trunk/initloma3/data/*.txt, list-directed y(1..my), main.f:726-727) for
tests/test_reference_meshes.py.

Source (read as text; nothing of the reference is executed):
  Beovulfo/LoMa_phD branches/reactml/benchmark_fft/cfttest_double.txt
  Beovulfo/LoMa_phD branches/reactml/benchmark_fft/rffttest_double.txt
written by branches/reactml/benchmark_fft/main.f:86-160 with Fortran format
5E14.7 (several values per record, no separators between negative numbers).

cfttest: triples (phys(k), Re fou(k), Im fou(k)), k=1..384: the rectangle
  function and its direct c2c transform (cft, iopt=-1, scaled by 1/n).
rffttest: pairs (physx(i), four(i)), i=1..768: four(1..768) is the packed
  direct real transform (rft, iopt=-1) of the rectangle four(257:511)=1 with
  four(385)=0.5 (main.f:128-138 sets four(k) with a stale index k=385, so the
  two 0.5 end values land on element 385 and elements 256/512 stay 0).
  physx(1) is overwritten by the transform's Nyquist slot (rft writes
  element n+1 past the 768-long array), so only four(:) is kept.

Usage: python tests/golden/make_golden.py <reference_root>
"""
import os
import sys

import numpy as np


# y meshes of the reference: a symmetric s = 8 mesh (453 points), the
# stretched mesh of the Pantano case (387) and an 801-point mesh whose last
# point stops short of symmetry
MESHES = ("meshs8Ly173", "pantanoBmy387", "LOMAmy801")


def parse_e14(path):
    vals = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            for i in range(0, len(line), 14):
                tok = line[i:i + 14].strip()
                if tok:
                    vals.append(float(tok))
    return np.array(vals)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference_root>  (the Beovulfo/LoMa_phD checkout)")
    root = sys.argv[1]
    d = os.path.join(root, "branches", "reactml", "benchmark_fft")
    c = parse_e14(os.path.join(d, "cfttest_double.txt")).reshape(-1, 3)
    r = parse_e14(os.path.join(d, "rffttest_double.txt")).reshape(-1, 2)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fft_rect_double.npz")
    np.savez(out, cft_phys=c[:, 0], cft_re=c[:, 1], cft_im=c[:, 2],
             rft_physx=r[:, 0], rft_four=r[:, 1])
    print("wrote", out, c.shape, r.shape)
    here = os.path.dirname(os.path.abspath(__file__))
    for code in ("lomacte3", "lomacte"):
        src = os.path.join(root, "trunk", code, "hre.dat")
        dst = os.path.join(here, f"hre_{code}.dat")
        with open(src, "rb") as f, open(dst, "wb") as g:
            g.write(f.read())
        print("wrote", dst)
    for name in MESHES:
        src = os.path.join(root, "trunk", "initloma3", "data", name + ".txt")
        dst = os.path.join(here, f"mesh_{name}.txt")
        with open(src, "rb") as f, open(dst, "wb") as g:
            g.write(f.read())
        print("wrote", dst)


if __name__ == "__main__":
    main()
