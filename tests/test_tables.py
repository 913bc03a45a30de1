"""The committed WENO tables are exactly what their generators produce, and
the product's rearranged tables agree with the oracle's direct forms."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _regen(script, committed):
    out = subprocess.run([sys.executable, script], stdout=subprocess.PIPE, check=True, text=True).stdout
    with open(committed) as f:
        assert f.read() == out


def test_oracle_tables_regenerate():
    _regen(os.path.join(ROOT, "oracle", "gen_tables.py"), os.path.join(ROOT, "oracle", "weno9_tables.h"))


def test_product_tables_regenerate():
    _regen(os.path.join(ROOT, "porturb_b200", "csrc", "gen_weno9.py"),
           os.path.join(ROOT, "porturb_b200", "csrc", "weno9_tables.cuh"))


def _parse_product_tables():
    txt = open(os.path.join(ROOT, "porturb_b200", "csrc", "weno9_tables.cuh")).read()
    env = {}
    for name in ("TV_D", "TV_L", "LIN_L", "LIN_R", "IDEAL_L", "IDEAL_R"):
        i = txt.index(name)
        body = txt[txt.index("=", i) + 1: txt.index(";", i)]
        env[name] = np.array(eval(body.replace("{", "[").replace("}", "]")))
    return env


def test_product_forms_match_direct_forms(oracle_lib):
    """TV and edge values from the product's difference/LDL^T tables equal the
    direct polynomial forms (evaluated by the oracle in FP64 with the ideal
    weights, i.e. linear reconstruction) on random stencils."""
    import pyoracle
    t = _parse_product_tables()
    rng = np.random.default_rng(3)
    for _ in range(100):
        s = rng.normal(size=9)
        d = np.diff(s)
        tv = []
        for k in range(5):
            y = [d[k + r] + sum(t["TV_L"][k][c][r] * d[k + c] for c in range(r + 1, 4)) for r in range(4)]
            tv.append(sum(t["TV_D"][k][r] * y[r] ** 2 for r in range(4)))
        eL = [s[4] + sum(t["LIN_L"][k][m] * d[k + m] for m in range(4)) for k in range(5)]
        eR = [s[4] + sum(t["LIN_R"][k][m] * d[k + m] for m in range(4)) for k in range(5)]
        # Weighted with the nonlinear weights of the oracle's own TVs, the edges must agree:
        tvn = np.array(tv) / sum(tv)
        wl = t["IDEAL_L"] / (tvn ** 2 + 1e-20)
        wr = t["IDEAL_R"] / (tvn ** 2 + 1e-20)
        qL = np.dot(wl / wl.sum(), eL)
        qR = np.dot(wr / wr.sum(), eR)
        oL, oR = pyoracle.weno9(s, False, False, False, kind="f64")
        assert abs(qL - oL) < 1e-9 * (1 + abs(oL)) and abs(qR - oR) < 1e-9 * (1 + abs(oR))
