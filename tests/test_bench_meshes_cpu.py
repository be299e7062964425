"""Two meshes of the reference's own benchmark (src/bench.sh:3; fixtures
copied by tests/golden/make_golden.py): E510, a soil trench of 510 boundary
and 5 enclosing elements, and Esoil_1600 (1600 + 5), NPG=8, one frequency,
L=76 interior points.  No outputs ship with them; these tests pin the
readers on the reference's own files (a tab before the frequency, records
spread over lines) and run the oracle on the second geometry class: its
solution satisfies its system and every reported number is finite."""
import os

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import formats, host

MESHES = {"E510": (515, 510, 555), "Esoil_1600": (1605, 1600, 1685)}


def _read(golden_dir, name):
    s = formats.read_static(os.path.join(golden_dir, f"{name}e.dat"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"{name}d.dat"), s.nbe)
    return s, d


@pytest.mark.parametrize("name", list(MESHES))
def test_reader_on_the_benchmark_meshes(golden_dir, name):
    s, d = _read(golden_dir, name)
    assert (s.n, s.nbe, s.np) == MESHES[name] and s.npg == 8
    assert (s.ge, s.rnu) == (1.0, 0.3)
    assert s.cone.min() == 1 and s.cone.max() == s.np
    assert (d.l, d.nfr, d.dam, d.rho) == (76, 1, 0.0, 1.0) and d.freqs.tolist() == [1.0]
    assert d.kode.shape == (3 * s.nbe,) and set(np.unique(d.kode)) <= {0, 1}
    assert d.cxi.shape == (76,) and np.all(np.isfinite(d.cxi))
    # the echoes the reference writes for them come out whole
    e = formats.format_static_echo(s).split("\n")
    assert len(e) == 19 + s.np + 5 + s.n + 1
    h = formats.format_dynamic_echo(s, d, host.material(s.ge, s.rnu, d.dam, d.rho)).split("\n")
    assert h[-1] == "" and h[-2].startswith("     76")


def test_oracle_on_the_soil_trench(golden_dir):
    s, d = _read(golden_dir, "E510")
    p = oracle.OracleProblem(s, d)
    hd, gd, _ = p.ghmatece()
    assert np.all(np.isfinite(hd)) and np.all(np.isfinite(gd))
    fr = float(d.freqs[0])
    zh, zfi, _, _ = p.system(fr)
    disp, trac, x = p.solve(fr, use_openblas=True)
    a = zh.reshape(p.nn, p.nn, order="F")
    assert np.linalg.norm(a @ x - zfi) <= 1e-12 * np.linalg.norm(zfi)
    zdsol, zssol = p.interior(fr, disp, trac)
    assert zdsol.shape == (3 * 76,) and zssol.shape == (9 * 76,)
    assert np.all(np.isfinite(zdsol)) and np.all(np.isfinite(zssol))
    # the traction-loaded trench moves: a nonzero, finite response
    assert 0.0 < np.abs(disp).max() < 1e6
