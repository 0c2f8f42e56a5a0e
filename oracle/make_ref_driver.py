"""Recipe: a Python-3 copy of the reference's MD driver, for the drop-in test.

TEST INFRASTRUCTURE ONLY. The reference's driver, yukawa_MD_p3m_ord6.py, is a
Python-2 script whose only Python-2 construct is the print statement
(yukawa_MD_p3m_ord6.py:81-95,123,145,152,175-176,186,193,203,246-251). This
recipe rewrites each ``print a, b`` as ``print(a, b)`` and changes nothing
else: same imports (read, initialize_pos_vel, velocity_verlet_p3m_ord6,
thermostat_p3m_ord6, yukawa_gf_opt, yukawa_p3m_ord6), same hand-set P3M
parameters, same loops and files. Run with this package's directory first on
``sys.path``, the copy calls this package's modules of those names -- the
drop-in boundary -- exactly as the reference's driver calls the reference's.

The output goes to ``oracle/_ref/`` (git-ignored, like the compiled reference
PP routine), never into the repository's history:

    python oracle/make_ref_driver.py <reference tree> [<output dir>]
"""
from __future__ import annotations

import os
import re
import sys

_PRINT = re.compile(r"^(\s*)print\s+(?!\()(.*)$")
NAME = "yukawa_MD_p3m_ord6.py"
OUT_NAME = "yukawa_MD_p3m_ord6_py3.py"


def convert(src: str) -> str:
    """Rewrite Python-2 print statements as calls; every other line as is."""
    return "\n".join(_PRINT.sub(r"\1print(\2)", ln) for ln in src.splitlines()) + "\n"


def main(argv):
    if len(argv) < 1:
        raise SystemExit("usage: make_ref_driver.py <reference tree> [<output dir>]")
    ref = argv[0]
    out_dir = argv[1] if len(argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                          "_ref")
    src_path = os.path.join(ref, NAME)
    if not os.path.isfile(src_path):
        print(f"{src_path} absent: skipping the driver copy")
        return
    with open(src_path) as f:
        text = convert(f.read())
    compile(text, OUT_NAME, "exec")  # must be valid Python 3
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, OUT_NAME), "w") as f:
        f.write(text)


if __name__ == "__main__":
    main(sys.argv[1:])
