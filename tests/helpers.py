"""Shared test helpers: case construction and golden loading."""
import os

import numpy as np
import yaml

from conftest import GOLDEN

CASE_TMPL = {
    "case": "cavity_test",
    "domain": {"lx": 1.0, "ly": 1.0, "lz": 1.0},
    "grid": {"nx": 24, "ny": 24, "nz": 24},
    "physics": {"reynolds": 400, "sgs": {"enabled": True, "model": "wale", "cw": 0.46}},
    "initial": {"type": "rest", "noise": 0.01},
    "boundaries": {"west": "wall", "east": "wall", "south": "slip", "north": "slip",
                   "bottom": "wall", "top": "moving_lid", "lid_velocity": 1.0},
    "numerics": {"mg_levels": 3, "max_outer_iters": 30, "div_tolerance": 1.0e-6},
    "time": {"n_steps": 30, "variable_dt": True, "dt_init": 3.0e-4,
             "safety_factor": 0.8, "dt_growth": 1.1},
    "output": {"n_out": 1000, "log_interval": 10, "outdir": "/tmp/warpflow_test"},
    "mpi": {"domains": [1, 1, 1]},
}


def make_cfg(n=24, levels=3, re=400.0, sgs=True, noise=0.01, ulid=1.0, vdt=True,
             dt0=3.0e-4, maxcy=30, precision="fp64"):
    from warpflow.config import case_from_dict
    raw = yaml.safe_load(yaml.safe_dump(CASE_TMPL))
    raw["grid"] = {"nx": n, "ny": n, "nz": n}
    raw["numerics"]["mg_levels"] = levels
    raw["numerics"]["max_outer_iters"] = maxcy
    raw["numerics"]["mg_precision"] = precision
    raw["physics"]["reynolds"] = re
    raw["physics"]["sgs"]["enabled"] = sgs
    raw["initial"]["noise"] = noise
    raw["boundaries"]["lid_velocity"] = ulid
    raw["time"]["variable_dt"] = vdt
    raw["time"]["dt_init"] = dt0
    return case_from_dict(raw)


def golden(tag):
    return np.load(os.path.join(GOLDEN, "golden_%s.npz" % tag))


def golden_cfg(g):
    from warpflow.config import case_from_dict
    return case_from_dict(yaml.safe_load(str(g["case_yaml"])))


GOLDEN_CAVITY = ["c8_l3_vdt", "c12_l3_fdt_re100", "c8_l2_nosgs", "c16_l3_vdt"]
