"""athinput blocks for the reference's three problem generators at the sizes
this project measures and tests (reference athinput.blast / .cpaw2d /
.field_loop, with gamma written as 5/3 to full precision).
"""
from __future__ import annotations

import math

GAMMA = 1.6666666666666667


def _grid(nx1, nx2, x1, x2, bc):
    ix1, ox1, ix2, ox2 = bc
    return {"Nx1": nx1, "x1min": x1[0], "x1max": x1[1], "ibc_x1": ix1, "obc_x1": ox1,
            "Nx2": nx2, "x2min": x2[0], "x2max": x2[1], "ibc_x2": ix2, "obc_x2": ox2}


def blast(nx1=200, nx2=300, tlim=0.2, bc=(4, 4, 4, 4), nlim=100000, flux="roe",
          prat=100.0, radius=0.1, b0=1.0, angle=45.0, pamb=0.1, cour_no=0.8):
    """MHD blast: [-0.5,0.5] x [-0.75,0.75] (src/blast.c:25-72)."""
    half = 0.5 * nx2 / nx1  # domain aspect = nx1:nx2 (200x300 -> +-0.75)
    return {
        "job": {"problem_id": "Blast", "maxout": 0, "flux": flux},
        "time": {"cour_no": cour_no, "nlim": nlim, "tlim": tlim},
        "grid": _grid(nx1, nx2, (-0.5, 0.5), (-half, half), bc),
        "problem": {"gamma": GAMMA, "pamb": pamb, "prat": prat, "b0": b0,
                    "radius": radius, "angle": angle},
    }


CPAW_PERIOD = 1.0 / math.sqrt(5.0)  # wavelength 1/sqrt(5), v_A = 1


def cpaw2d(nx1=64, nx2=32, tlim=CPAW_PERIOD, flux="roe", nlim=100000, cour_no=0.8):
    """Circularly polarised Alfven wave on [0,1] x [0,0.5], k = 2 pi (1,2)
    (src/cpaw2d.c:56-185; the angle becomes atan(2) for this box)."""
    return {
        "job": {"problem_id": "cpaw", "maxout": 0, "flux": flux},
        "time": {"cour_no": cour_no, "nlim": nlim, "tlim": tlim},
        "grid": _grid(nx1, nx2, (0.0, 1.0), (0.0, 0.5), (4, 4, 4, 4)),
        "problem": {"gamma": GAMMA, "angle": 63.4, "pres": 0.1, "v_par": 0.0,
                    "b_par": 1.0, "b_perp": 0.1},
    }


def field_loop(nx1=1024, nx2=512, tlim=1.0, flux="roe", nlim=100000, cour_no=0.8,
               bc=(4, 4, 4, 4)):
    """Field-loop advection on [-1,1] x [-0.5,0.5] with v = (2,1)
    (src/field_loop.c:40-137; vflow = sqrt(5) gives v = (2, 1))."""
    return {
        "job": {"problem_id": "Loop", "maxout": 0, "flux": flux},
        "time": {"cour_no": cour_no, "nlim": nlim, "tlim": tlim},
        "grid": _grid(nx1, nx2, (-1.0, 1.0), (-0.5, 0.5), bc),
        "problem": {"gamma": GAMMA, "rad": 0.3, "amp": 1.0e-3,
                    "vflow": 2.23606797749979, "iprob": 1},
    }


BUILDERS = {"blast": blast, "cpaw2d": cpaw2d, "field_loop": field_loop}
