"""The reference's golden-file checker (src/dtester.c), compiled into
oracle/_ref/dtester by `make -C oracle ref`, run on a dynamic output file
written the way the reference writes it (formats.write_dynamic_output:
INPUTECD's echo, from which the checker reads the mesh sizes, then the
OUTPUTEC result block)."""
import os
import re
import subprocess

from bem_mececcs_b200 import formats, host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DTESTER = os.path.join(ROOT, "oracle", "_ref", "dtester")
ENC = "latin-1"
KEYS = ("disp", "traction", "idisp", "sigma")


def available() -> bool:
    return os.access(DTESTER, os.X_OK)


def build() -> bool:
    """Builds the checker where the reference tree is present; True if it exists."""
    if not available():
        import __graft_entry__
        ref = __graft_entry__.reference_tree()
        if ref:
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref}"],
                           capture_output=True)
    return available()


def write(path: str, s, d, res: "formats.Results") -> None:
    """The output file of the run (s, d) whose only frequency gave `res`."""
    formats.write_dynamic_output(path, s, d, host.material(s.ge, s.rnu, d.dam, d.rho), [res])


def run(ours: str, gold_path: str):
    """(exit status, the four errors the checker prints)."""
    p = subprocess.run([DTESTER, ours, gold_path], capture_output=True, text=True, encoding=ENC)
    vals = [float(v) for v in re.findall(r":\s*([-+0-9.E]+)\s*$", p.stdout, re.M)]
    if len(vals) != 4:
        raise AssertionError(f"unexpected checker output: {p.stdout!r} {p.stderr!r}")
    return p.returncode, dict(zip(KEYS, vals))


def check_run(s, d, res: "formats.Results", gold_path: str, workdir: str):
    """Writes the output file of the run (s, d) and runs the checker on it.
    Returns (exit status, the checker's four errors, formats.dtester_errors
    on the same two files).  The file holds 4 printed digits, so the last two
    agree with each other, not with the metric taken on `res` in memory."""
    ours = os.path.join(workdir, "ours_" + os.path.basename(gold_path))
    write(ours, s, d, res)
    rc, ref_err = run(ours, gold_path)
    file_err = formats.dtester_errors(formats.parse_results(ours)[0],
                                      formats.parse_results(gold_path)[0])
    return rc, ref_err, file_err


def result_block(gold_path: str) -> str:
    """The golden file's result block, from its frequency line to the end."""
    lines = open(gold_path, encoding=ENC).read().split("\n")
    i = next(k for k, ln in enumerate(lines) if "FREQ\xdc\xcaNCIA =" in ln)
    return "\n".join(lines[i - 3:])
