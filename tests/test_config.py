"""The JSON front end (the reference's case-file format,
Src/configuration.cpp:152-223): round trips of every case builder and of
the random cases, dump/load through a file, the reference's own app files,
and rejection of what the path does not run."""
import dataclasses

import pytest

import golden_cases
import random_cases
from mplb_b200 import config

BUILDERS = {
    "cavity2d": lambda: config.cavity(2, 9, 0.05, re=100),
    "cavity3d_order": lambda: config.cavity(
        3, 7, 0.05, re=100, order=("Front", "Left", "Right", "Top", "Bottom",
                                   "Back")),
    "cavity3d_fp16": lambda: config.cavity(3, 7, 0.05, re=100,
                                           precision="fp16"),
    "cavity3d_swap": lambda: config.cavity(
        3, 7, 0.05, re=100, scheme="Scheme_StreamCollision_Swap"),
    "poiseuille2d": lambda: config.poiseuille(2, 8, 6),
    "poiseuille3d_bb": lambda: config.poiseuille(3, 6, 6, 5,
                                                 wall="HalfwayBounceBack"),
    "lchannel": lambda: config.lchannel(leg=12, side=8, depth=6),
    "lchannel_app": lambda: config.lchannel_app(9),
}
for _s in random_cases.SEEDS[:8]:
    BUILDERS[f"random{_s}"] = lambda s=_s: random_cases.random_case(s)[0]
for _s in random_cases.MULTI_SEEDS[:4]:
    BUILDERS[f"two_blocks{_s}"] = (
        lambda s=_s: random_cases.random_two_blocks(s)[0])
for _s in random_cases.SWAP_SEEDS[:4]:
    BUILDERS[f"swap{_s}"] = lambda s=_s: random_cases.random_swap_box(s)[0]


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_round_trip(name, tmp_path):
    case = BUILDERS[name]()
    js = case.to_json()
    back = config.CaseConfig.from_json(js)
    assert back.to_json() == js
    for f in ("space_dim", "block_ids", "block_sizes", "boundaries",
              "connections", "force_velocity", "body_force", "scheme",
              "precision", "initial"):
        assert getattr(back, f) == getattr(case, f), f
    path = tmp_path / "case.json"
    case.dump(str(path))
    assert config.CaseConfig.load(str(path)).to_json() == js


def test_swap_names_carry_the_suffix():
    js = BUILDERS["cavity3d_swap"]().to_json()
    assert js["CollisionType"] == ["Collision_BGKIsothermal2nd_Swap"]
    assert js["BodyForceType"] == ["BodyForce_None_Swap"]
    assert config.CaseConfig.from_json(js).body_force == "BodyForce_None"


def test_reference_app_files_parse():
    apps = golden_cases.apps()
    assert len(apps) == 3
    for name, (case, steps, _) in apps.items():
        assert steps > 0
        assert config.CaseConfig.from_json(case.to_json()).to_json() == \
            case.to_json(), name


def _edit(**kw):
    js = config.cavity(3, 7, 0.05, re=100).to_json()
    js.update(kw)
    return js


@pytest.mark.parametrize("js,words", [
    (_edit(CompoNames=["A", "B"]), "one component"),
    (_edit(LatticeName=["d3q15"]), "lattice"),
    (_edit(LatticeName=["d2q9"]), "lattice"),
    (_edit(SchemeType="Scheme_Unknown"), "scheme"),
    (_edit(CollisionType=["Collision_BGKThermal4th"]), "collision"),
    (_edit(CollisionType=["Collision_BGKIsothermal2nd_Swap"]), "collision"),
    (_edit(BodyForceType=["BodyForce_2nd"]), "body force"),
    (_edit(SchemeType="Scheme_StreamCollision_Swap"), "collision"),
])
def test_rejects(js, words):
    with pytest.raises(ValueError, match=words):
        config.CaseConfig.from_json(js)


def test_force_velocity_from_macro_types():
    case = config.poiseuille(3, 6, 6, 5)
    js = case.to_json()
    assert js["MacroVarTypes"][1:] == ["Variable_U_Force", "Variable_V_Force",
                                       "Variable_W_Force"]
    assert config.CaseConfig.from_json(js).force_velocity
    plain = dataclasses.replace(case, force_velocity=False).to_json()
    assert not config.CaseConfig.from_json(plain).force_velocity
