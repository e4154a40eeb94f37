"""Case loading and topology (host logic, reference config.py / topology.py)."""
import pytest
import yaml

from helpers import CASE_TMPL, make_cfg


def test_load_reference_style_case(tmp_path):
    from warpflow.config import load_case
    p = tmp_path / "c.yaml"
    p.write_text(yaml.safe_dump(CASE_TMPL))
    cfg = load_case(p)
    assert cfg.name == "cavity_test"
    assert cfg.grid.nx == 24 and cfg.numerics.mg_levels == 3
    assert cfg.physics.sgs_enabled and cfg.physics.sgs_cw == 0.46
    assert cfg.boundaries.top == "moving_lid"
    assert cfg.numerics.mg_precision == "fp64"


def test_divisibility_errors():
    with pytest.raises(ValueError, match="divisible by 2\\*\\*\\(mg_levels-1\\)=4"):
        make_cfg(n=10, levels=3)


def test_unknown_key_rejected():
    from warpflow.config import case_from_dict
    raw = yaml.safe_load(yaml.safe_dump(CASE_TMPL))
    raw["numerics"]["bogus"] = 1
    with pytest.raises(TypeError):
        case_from_dict(raw)


def test_precision_key():
    assert make_cfg(precision="mixed").numerics.mg_precision == "mixed"
    with pytest.raises(ValueError):
        make_cfg(precision="fp16")


def test_single_rank_topology():
    from warpflow.topology import build_topology
    cfg = make_cfg(n=16)
    t = build_topology(cfg)
    assert t.rank == 0 and t.nranks == 1
    assert t.local_ncells == (16, 16, 16)
    assert all(v == (-1, -1) for v in t.neighbors.values())
    assert t.comm.allreduce(3.5) == 3.5
    cfg.mpi.domains = (2, 1, 1)
    with pytest.raises(ValueError, match="implies 2 ranks"):
        build_topology(cfg)


def test_boundary_combination_checked():
    from warpflow.bcs import BoundaryKernels
    bnd = {"west": "wall", "east": "wall", "south": "slip", "north": "slip",
           "bottom": "wall", "top": "moving_lid"}
    BoundaryKernels(bnd, "cuda:0")
    bnd["north"] = "periodic"
    with pytest.raises(ValueError, match="unsupported boundary combination"):
        BoundaryKernels(bnd, "cuda:0")


def test_cpu_device_refused():
    """No CPU fallback: asking for device='cpu' fails loudly."""
    from warpflow.fields import cuda_device
    with pytest.raises(RuntimeError, match="CUDA devices only"):
        cuda_device("cpu")
