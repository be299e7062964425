"""Copies the reference's known-answer fixtures into tests/golden/.

The reference pins its hot path end to end with two meshes (src/tests.sh:38-117):
ESOLO240 (N=240, NBE=100) and ESOLO2160 (N=2160, NBE=900), NPG=8, nu=0.3,
omega=1, L=10 interior points.  The golden dynamic outputs SSOLO*D were
printed with D11.4 (src/Outputec.for:37) and are checked by src/dtester.c at
EPS=1e-3; the static outputs SSOLO*E (the input echo with the element
centroids, src/Inputece.for:29-104) must match byte for byte
(src/tests.sh:43).  These data files are copied verbatim (they are inputs and
outputs, not source); run this script in a container where the reference is
mounted.

Two of the meshes of the reference's own benchmark (src/bench.sh:3, inputs
only, from malhas.zip at the reference's root) are copied too: E510 (a soil
trench, 510 boundary + 5 enclosing elements) and Esoil_1600 (1600 + 5), both
NPG=8 with L=76 interior points.  They carry no shipped outputs; they pin the
readers on the reference's own files and give the oracle (and the GPU) a
second geometry class.
"""
import hashlib
import os
import shutil
import sys
import zipfile

# The reference's src/ directory: the first argument, else BEM_REFERENCE_TREE/src.
SRC = (sys.argv[1] if len(sys.argv) > 1 else
       os.path.join(os.environ["BEM_REFERENCE_TREE"], "src") if "BEM_REFERENCE_TREE" in os.environ else None)
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ["ESOLO240E_-5+5.DAT", "ESOLO240D_-5+5.DAT", "SSOLO240D_-5+5.SOL",
         "ESOLO2160E_-5+5.DAT", "ESOLO2160D_-5+5.DAT", "SSOLO2160D_-5+5.SOL",
         "SSOLO240E_-5+5.SOL", "SSOLO2160E_-5+5.SOL"]
ZIPPED = ["E510e.dat", "E510d.dat", "Esoil_1600e.dat", "Esoil_1600d.dat"]

if __name__ == "__main__":
    if SRC is None:
        sys.exit("usage: make_golden.py <reference>/src  (or set BEM_REFERENCE_TREE)")
    with open(os.path.join(HERE, "SHA256SUMS"), "w") as out:
        for f in FILES:
            dst = os.path.join(HERE, f)
            shutil.copyfile(os.path.join(SRC, f), dst)
            with open(dst, "rb") as fh:
                out.write(f"{hashlib.sha256(fh.read()).hexdigest()}  {f}\n")
        with zipfile.ZipFile(os.path.join(SRC, os.pardir, "malhas.zip")) as z:
            for f in ZIPPED:
                data = z.read(f)
                with open(os.path.join(HERE, f), "wb") as fh:
                    fh.write(data)
                out.write(f"{hashlib.sha256(data).hexdigest()}  {f}\n")
    print("copied", len(FILES) + len(ZIPPED), "fixtures")
