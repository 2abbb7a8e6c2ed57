"""Descriptor validation of mplbgpu_create, which runs before the device is
looked for: every rejection the plan builder makes (plan.cpp) with its
status and message, and acceptance of every case the parity tests use
(without a GPU an accepted description ends in MPLBGPU_ERR_NO_DEVICE)."""
import ctypes
import dataclasses

import pytest

import golden_cases
import random_cases
import special_cases
from mplb_b200 import abi, build, config


@pytest.fixture(scope="module")
def lib():
    build.build()
    return abi.load_library()


def create(lib, case, edit=None):
    d, keep = case.to_desc()
    if edit:
        edit(d)
    h = ctypes.c_void_p()
    rc = lib.mplbgpu_create(ctypes.byref(d), ctypes.byref(h))
    msg = lib.mplbgpu_last_error(None).decode()
    if rc == abi.OK:
        lib.mplbgpu_destroy(h)
    return rc, msg


def accepted(rc):
    return rc in (abi.OK, abi.ERR_NO_DEVICE)


def cav3(**kw):
    return config.cavity(3, 6, 0.05, re=100, **kw)


def cav2(**kw):
    return config.cavity(2, 6, 0.05, re=100, **kw)


def swap3(**kw):
    return config.cavity(3, 6, 0.05, re=100,
                         scheme="Scheme_StreamCollision_Swap", **kw)


def two_blocks():
    case, _ = random_cases.random_two_blocks(1)
    return case


def set_attr(name, value):
    return lambda d: setattr(d, name, value)


def set_block(i, **kw):
    def f(d):
        for k, v in kw.items():
            if k == "size":
                for a in range(3):
                    d.blocks[i].size[a] = v[a]
            else:
                setattr(d.blocks[i], k, v)
    return f


def set_bc(i, **kw):
    def f(d):
        for k, v in kw.items():
            setattr(d.boundaries[i], k, v)
    return f


def set_conn(i, **kw):
    def f(d):
        for k, v in kw.items():
            setattr(d.connections[i], k, v)
    return f


def with_cut(case, cut):
    return dataclasses.replace(case, cuts={0: cut})


S = abi.SURFACES
REJECTED = {
    "abi_version": (cav3, set_attr("abi_version", 99), abi.ERR_INVALID,
                    "abi_version"),
    "lattice_of_other_dim": (cav2, set_attr("lattice", 19),
                             abi.ERR_UNSUPPORTED, "D2Q9"),
    "precision": (cav3, set_attr("precision", 7), abi.ERR_INVALID,
                  "precision"),
    "no_blocks": (cav3, set_attr("nblocks", 0), abi.ERR_INVALID, "no blocks"),
    "tau": (cav3, set_attr("tau_ref", -1.0), abi.ERR_INVALID, "positive"),
    "dt": (cav3, set_attr("dt", 0.0), abi.ERR_INVALID, "positive"),
    "body_force": (cav3, set_attr("body_force", 5), abi.ERR_UNSUPPORTED,
                   "body force"),
    "scheme": (cav3, set_attr("scheme", 12), abi.ERR_UNSUPPORTED, "scheme"),
    "swap_2d": (lambda: config.cavity(2, 6, 0.05, re=100,
                                      scheme="Scheme_StreamCollision_Swap"),
                None, abi.ERR_UNSUPPORTED, "swap"),
    "swap_connections": (lambda: dataclasses.replace(
        config.poiseuille(3, 6, 6, 6), scheme="Scheme_StreamCollision_Swap"),
        None, abi.ERR_UNSUPPORTED, "swap"),
    "swap_two_nodes": (lambda: dataclasses.replace(
        swap3(), block_sizes=[(6, 2, 6)]), None, abi.ERR_UNSUPPORTED,
        "at least 3"),
    "swap_outlet": (swap3, set_bc(0, scheme=abi.BC_SCHEMES[
        "ExtrapolPressure1ST"], vertex_type=abi.VERTEX_TYPES["OutLet"]),
        abi.ERR_UNSUPPORTED, "node-local"),
    "duplicate_block": (two_blocks, set_block(1, id=0), abi.ERR_INVALID,
                        "duplicate"),
    "one_node_axis": (cav3, set_block(0, size=(6, 1, 6)), abi.ERR_INVALID,
                      "at least 2"),
    "cut_beyond_dim": (lambda: with_cut(cav2(), 1 << S["Front"]), None,
                       abi.ERR_INVALID, "cut faces"),
    "cut_with_connections": (lambda: dataclasses.replace(
        config.poiseuille(3, 6, 6, 6), cuts={0: 1 << S["Top"]}), None,
        abi.ERR_UNSUPPORTED, "cut"),
    "bc_on_cut_face": (lambda: with_cut(cav3(), 1 << S["Front"]), None,
                       abi.ERR_INVALID, "cut face"),
    "bc_unknown_block": (cav3, set_bc(2, block=7), abi.ERR_INVALID,
                         "unknown block"),
    "bc_surface_of_other_dim": (cav2, set_bc(1, surface=S["Front"]),
                                abi.ERR_INVALID, "surface"),
    "bc_surface_value": (cav3, set_bc(1, surface=99), abi.ERR_INVALID,
                         "surface"),
    "fdperiodic_swap": (swap3, set_bc(0, scheme=abi.BC_SCHEMES["FDPeriodic"]),
                        abi.ERR_UNSUPPORTED, "FDPeriodic"),
    "immersed_solid": (cav3, set_bc(3, vertex_type=abi.VERTEX_TYPES[
        "ImmersedSolid"]), abi.ERR_UNSUPPORTED, "immersed"),
    "connection_unknown_block": (two_blocks, set_conn(0, to_block=9),
                                 abi.ERR_INVALID, "unknown block"),
    "connection_surface_of_other_dim": (
        lambda: random_cases.random_two_blocks(0)[0],
        set_conn(0, from_surface=S["Front"]), abi.ERR_INVALID, "dimension"),
    "connected_sizes_differ": (two_blocks, set_block(1, size=(9, 9, 9)),
                               abi.ERR_INVALID, "differ in size"),
}


@pytest.mark.parametrize("name", sorted(REJECTED))
def test_rejected(lib, name):
    build_case, edit, code, words = REJECTED[name]
    rc, msg = create(lib, build_case(), edit)
    assert rc == code, (name, rc, msg)
    assert words.lower() in msg.lower(), (name, msg)


def accepted_cases():
    out = {name: (lambda n=name: golden_cases.load(n)["case"])
           for name in golden_cases.names(include_long=True)}
    for s in random_cases.SEEDS:
        out[f"random{s}"] = lambda s=s: random_cases.random_case(s)[0]
    for s in random_cases.MULTI_SEEDS:
        out[f"two_blocks{s}"] = lambda s=s: random_cases.random_two_blocks(s)[0]
    for s in random_cases.SWAP_SEEDS:
        out[f"swap{s}"] = lambda s=s: random_cases.random_swap_box(s)[0]
    for p in ("fp32", "fp16"):
        out[f"cavity3d_{p}"] = lambda p=p: cav3(precision=p)
        out[f"swap_{p}"] = lambda p=p: swap3(precision=p)
    out["lchannel_bb"] = lambda: config.lchannel(leg=9, side=6, depth=4,
                                                 wall="HalfwayBounceBack")
    out["fdperiodic"] = special_cases.fdperiodic_channel
    out["slab_middle"] = lambda: with_cut(
        dataclasses.replace(cav3(), boundaries=[
            b for b in cav3().boundaries
            if b.surface not in ("Front", "Back")]),
        (1 << S["Front"]) | (1 << S["Back"]))
    return out


ACCEPTED = accepted_cases()


@pytest.mark.parametrize("name", sorted(ACCEPTED))
def test_accepted(lib, name):
    rc, msg = create(lib, ACCEPTED[name]())
    assert accepted(rc), (name, rc, msg)


def test_reference_app_files_accepted(lib):
    apps = golden_cases.apps()
    assert apps
    for name, (case, _, _) in apps.items():
        rc, msg = create(lib, case)
        assert accepted(rc), (name, rc, msg)


def batch_create(lib, cavs, precision="fp32"):
    arr = (abi.Cavity * max(len(cavs), 1))()
    for i, (n, lid_u, tau_ref) in enumerate(cavs):
        arr[i].n, arr[i].lid_u, arr[i].tau_ref = n, lid_u, tau_ref
    h = ctypes.c_void_p()
    rc = lib.mplbgpu_batch_create(arr, len(cavs), abi.PRECISIONS[precision],
                                  ctypes.byref(h))
    msg = lib.mplbgpu_batch_last_error(None).decode()
    if rc == abi.OK:
        lib.mplbgpu_batch_destroy(h)
    return rc, msg


@pytest.mark.parametrize("cavs,precision,code,words", [
    ([], "fp32", abi.ERR_INVALID, "no cavities"),
    ([(64, 0.05, 0.01)], "fp16", abi.ERR_UNSUPPORTED, "FP64 or shifted FP32"),
    ([(64, 0.05, 0.01), (2, 0.05, 0.01)], "fp32", abi.ERR_INVALID,
     "cavity side"),
    ([(46341, 0.05, 0.01)], "fp64", abi.ERR_INVALID, "cavity side"),
    ([(64, 0.05, -1.0)], "fp32", abi.ERR_INVALID, "tau_ref"),
])
def test_batch_rejected(lib, cavs, precision, code, words):
    rc, msg = batch_create(lib, cavs, precision)
    assert rc == code and words in msg, (rc, msg)


def test_batch_accepted(lib):
    from mplb_b200.batch import cavity_set
    specs = cavity_set(64)
    cavs = [(s.n, 3 ** 0.5 * s.lid, s.tau_ref) for s in specs]
    for p in ("fp32", "fp64"):
        rc, msg = batch_create(lib, cavs, p)
        assert accepted(rc), (p, rc, msg)
