"""Initial states of case files of ours as the reference evaluates them (Simulation::initialize_field through
evaluate_initial, cpp/src/CaseFile.cpp:784-841, and its TinyExpr expressions), for tests/test_casefile.py.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_initial.py

Each case: a case file text of ours (background state, regions of every shape, expressions of the parameters and of the
cell centre) and parameter overrides; the reference (oracle/_ref, through oracle/ref/ref_harness.cpp's `case` key) sets
the run up from them and its initial state is stored in tests/golden/initial.npz. Test data only.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402

CASES = {
    "diaphragm_2d": ("""[case]
name = "init diaphragm"
description = "a diaphragm problem"

[initial]
state = { rho = 0.125, u = 0.0, v = 0.0, p = 0.1 }

[[initial.region]]
shape = "halfspace"
point = ["0.4*Lx", 0.0]
normal = [-1.0, 0.25]
state = { rho = 1.0, u = 0.3, p = "1.0 + 0.5*u_in" }
""", dict(nx=50, ny=12, Lx=1.0, Ly=0.2, u_in=0.8, bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall")),
    "box_sphere_3d": ("""[case]
name = "init box and sphere"
description = "regions in 3-D"

[initial]
state = { rho = "1.0 + 0.5*x/Lx - 0.25*y*z", u = 0.1, v = "-0.2", w = "0.05*z", p = "1/(gamma - 1)" }

[[initial.region]]
shape = "box"
min = ["Lx/3", 0.1]
max = ["2*Lx/3", "0.9*Ly"]
state = { rho = 2.0, p = "3^2^0.5" }

[[initial.region]]
shape = "sphere"
center = ["Lx/2", "Ly/2", "Lz/2"]
radius = "0.2*Lx"
state = { p = 10.0, u = "-(0.5 - 1.5)" }
""", dict(nx=14, ny=12, nz=10, Lx=2.0, Ly=1.0, Lz=1.5)),
    "box_sphere_3d_case": ("""[case]
name = "init box and sphere 3-D"
description = "regions of a 3-D case"
requires_3d = true

[initial]
state = { rho = "1.0 + 0.5*x/Lx - 0.25*y*z", u = 0.1, v = "-0.2", w = "0.05*z", p = "1/(gamma - 1)" }

[[initial.region]]
shape = "box"
min = ["Lx/3", 0.1, 0.2]
max = ["2*Lx/3", "0.9*Ly"]
state = { rho = 2.0, p = "3^2^0.5" }

[[initial.region]]
shape = "sphere"
center = ["Lx/2", "Ly/2", "Lz/2"]
radius = "0.2*Lx"
state = { p = 10.0, u = "-(0.5 - 1.5)" }
""", dict(nx=14, ny=12, nz=10, Lx=2.0, Ly=1.0, Lz=1.5)),
    "cylinder_trig_3d": ("""[case]
name = "init cylinder"
description = "a cylinder region and a periodic background"
requires_3d = true

[initial]
state = { rho = "1.0 + 0.1*sin(2*pi*x/Lx)*cos(2*pi*y/Ly)", u = "sqrt(2)*cos(pi*z)", v = 0.0, p = "1.0 + exp(-x)" }

[[initial.region]]
shape = "cylinder"
axis = "x"
center = [0.0, "Ly/2", "Lz/2"]
radius = 0.3
state = { rho = "2.0 + atan2(y, z)", w = "pow(abs(y - 0.5), 1.5)" }
""", dict(nx=10, ny=16, nz=12, Lx=1.0, Ly=1.0, Lz=1.0)),
    "stiffened_logs_2d": ("""[case]
name = "init stiffened"
description = "stiffened gas, logarithms and powers"

[initial]
state = { rho = 1000.0, u = 0.0, v = 0.0, p = "2^3 + ln(2) + log(100) + 7 % 3" }

[[initial.region]]
shape = "box"
min = [0.0, 0.0]
max = ["0.5*Lx", "Ly"]
state = { rho = 1.2, p = "-2^2 + 100000" }
""", dict(nx=20, ny=8, Lx=1.0, Ly=0.4, eos_type="Stiffened Gas", gamma=4.4, p_inf=6000.0)),
}


def main():
    out = {}
    for name, (text, over) in CASES.items():
        tmp = tempfile.mkdtemp(prefix="fvg_init_")
        path = os.path.join(tmp, "case.toml")
        with open(path, "w") as f:
            f.write(text)
        ref = Reference(dict(over, case=path))
        out[f"{name}/case_toml"] = np.array(text)
        out[f"{name}/overrides"] = np.array(json.dumps(over))
        out[f"{name}/U0"] = ref.state()
        print(f"{name}: {ref.state().shape[0]} cells")
    np.savez_compressed(os.path.join(HERE, "initial.npz"), **out)


if __name__ == "__main__":
    main()
