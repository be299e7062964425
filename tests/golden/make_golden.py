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
"""
import hashlib
import os
import shutil
import sys

SRC = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src"
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ["ESOLO240E_-5+5.DAT", "ESOLO240D_-5+5.DAT", "SSOLO240D_-5+5.SOL",
         "ESOLO2160E_-5+5.DAT", "ESOLO2160D_-5+5.DAT", "SSOLO2160D_-5+5.SOL",
         "SSOLO240E_-5+5.SOL", "SSOLO2160E_-5+5.SOL"]

if __name__ == "__main__":
    with open(os.path.join(HERE, "SHA256SUMS"), "w") as out:
        for f in FILES:
            dst = os.path.join(HERE, f)
            shutil.copyfile(os.path.join(SRC, f), dst)
            with open(dst, "rb") as fh:
                out.write(f"{hashlib.sha256(fh.read()).hexdigest()}  {f}\n")
    print("copied", len(FILES), "fixtures")
