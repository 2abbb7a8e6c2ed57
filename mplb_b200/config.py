"""Case descriptions in the reference's JSON configuration format.

``CaseConfig`` holds what MPLB's setup API holds after ``Partition()`` for a
single-component BGK case: blocks (DefineBlocks), connections
(DefineBlockConnection), the boundary list in definition order
(DefineBlockBoundary), lattice, tauRef, body force and the time step
``dt = MeshSize / SoundSpeed()``.  It reads and writes the reference's JSON
keys (Src/configuration.cpp:152-223, e.g. Apps/3DCavity/Cavity3D.json) plus
three keys the reference leaves to app code:

* ``InitialMacroVars``: {"rho": r, "u": u, "v": v, "w": w} uniform start
  (the apps' KerSetInitialMacroVars, Apps/3DCavity/cavity3d_kernel.inc);
* ``BodyAcceleration``: [ax, ay(, az)] uniform body acceleration (the apps'
  UpdateMacroscopicBodyForce hook);
* ``Precision``: "fp64" (default), "fp32" or "fp16" storage form.

Builders for the benchmark workloads are at the bottom: lattice-unit inputs
(lid speed, Re, tau) are converted to MPLB units with dx = 1/(N-1),
dt = dx/sqrt(3), tauRef = (tau_L - 1/2) dt, u_MPLB = sqrt(3) u_L
(Src/model.cpp:67-68, Src/model_kernel.inc:428-435).
"""
import ctypes
import dataclasses
import json
import math
from typing import Dict, List, Optional, Tuple

from . import abi

SQRT3 = math.sqrt(3.0)


@dataclasses.dataclass
class BoundaryDef:
    block: int
    surface: str
    scheme: str
    vertex_type: str = "Wall"
    given: Tuple[float, ...] = ()
    macro_types: Tuple[str, ...] = ()


@dataclasses.dataclass
class ConnectionDef:
    from_block: int
    from_surface: str
    to_block: int
    to_surface: str
    type: str


@dataclasses.dataclass
class CaseConfig:
    case_name: str
    space_dim: int
    block_ids: List[int]
    block_names: List[str]
    block_sizes: List[Tuple[int, ...]]
    mesh_size: float
    tau_ref: float
    boundaries: List[BoundaryDef]
    connections: List[ConnectionDef] = dataclasses.field(default_factory=list)
    start_pos: Optional[Dict[int, List[float]]] = None
    force_velocity: bool = False
    body_force: str = "BodyForce_None"
    accel: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    initial: Tuple[float, float, float, float] = (1.0, 0.0, 0.0, 0.0)
    check_period: int = 1000
    transient: bool = False
    convergence: float = 1e-8
    steps: int = 0
    precision: str = "fp64"
    scheme: str = "Scheme_StreamCollision"
    # decomposition (not part of the reference's JSON): per block id, bit s
    # set when surface s is cut, i.e. continues in another context
    cuts: Optional[Dict[int, int]] = None

    @property
    def swap(self) -> bool:
        return self.scheme == "Scheme_StreamCollision_Swap"

    @property
    def lattice(self) -> int:
        return abi.D2Q9 if self.space_dim == 2 else abi.D3Q19

    @property
    def q(self) -> int:
        return self.lattice

    @property
    def cs(self) -> float:
        return SQRT3

    @property
    def dt(self) -> float:
        return self.mesh_size / self.cs

    def nodes(self) -> int:
        return sum(math.prod(s) for s in self.block_sizes)

    def size3(self, block_id: int) -> Tuple[int, int, int]:
        s = self.block_sizes[self.block_ids.index(block_id)]
        return (s[0], s[1], s[2] if len(s) > 2 else 1)

    # -- reference JSON -------------------------------------------------
    def to_json(self) -> dict:
        d = self.space_dim
        mv = ["Variable_Rho", "Variable_U", "Variable_V", "Variable_W"][:d + 1]
        if self.force_velocity:
            mv = [mv[0]] + [m + "_Force" for m in mv[1:]]
        names = ["rho", "u", "v", "w"][:d + 1]
        # the swap scheme runs with the _Swap collision and body-force types
        # (Apps/3DCavity-Swap/lbm3d_cavity_swap.cpp:72-106)
        sfx = "_Swap" if self.swap else ""
        out = {
            "CaseName": self.case_name,
            "SpaceDim": d,
            "Transient": self.transient,
            "BlockIds": list(self.block_ids),
            "BlockNames": list(self.block_names),
            "BlockSize": [int(v) for s in self.block_sizes for v in s],
            "MeshSize": self.mesh_size,
            "StartPos": {str(i): list(p) for i, p in self._start_pos().items()},
            "CompoNames": ["Fluid"],
            "CompoIds": [0],
            "LatticeName": ["d2q9" if d == 2 else "d3q19"],
            "TauRef": [self.tau_ref],
            "MacroVarNames": names,
            "MacroVarIds": list(range(d + 1)),
            "MacroCompoIds": [0] * (d + 1),
            "MacroVarTypes": mv,
            "CollisionType": ["Collision_BGKIsothermal2nd" + sfx],
            "CollisionCompoIds": [0],
            "InitialType": ["Initial_BGKFeq2nd"],
            "InitialCompoIds": [0],
            "BodyForceType": [self.body_force + sfx],
            "BodyForceCompoId": [0],
            "SchemeType": self.scheme,
            "CurrentTimeStep": 0,
            "CheckPeriod": self.check_period,
            "ConvergenceCriteria": self.convergence,
            "TimeStepsToRun": self.steps,
            "InitialMacroVars": dict(zip(["rho", "u", "v", "w"],
                                         self.initial)),
            "BodyAcceleration": list(self.accel[:d]),
            "Precision": self.precision,
        }
        if self.connections:
            out["FromBlockIds"] = [c.from_block for c in self.connections]
            out["ToBlockIds"] = [c.to_block for c in self.connections]
            out["FromBoundarySurface"] = [c.from_surface
                                          for c in self.connections]
            out["ToBoundarySurface"] = [c.to_surface for c in self.connections]
            out["BlockConnectionType"] = [c.type for c in self.connections]
        for i, b in enumerate(self.boundaries):
            out[f"BoundaryCondition{i}"] = {
                "BlockIndex": b.block,
                "ComponentId": 0,
                "GivenVars": list(b.given),
                "BoundarySurface": b.surface,
                "BoundaryScheme": ("EQMDiffuseREfl"
                                   if b.scheme in ("EQMDiffuseRefl",
                                                   "EQMDiffuseREfl")
                                   else b.scheme),
                "BoundaryType": b.vertex_type,
                "MacroVarTypesatBoundary": list(b.macro_types),
            }
        return out

    def _start_pos(self) -> Dict[int, List[float]]:
        if self.start_pos:
            return self.start_pos
        return {i: [0.0] * self.space_dim for i in self.block_ids}

    @classmethod
    def from_json(cls, js: dict) -> "CaseConfig":
        d = int(js["SpaceDim"])
        ids = [int(v) for v in js["BlockIds"]]
        sizes = js["BlockSize"]
        block_sizes = [tuple(int(v) for v in sizes[i * d:(i + 1) * d])
                       for i in range(len(ids))]
        if len(js.get("CompoNames", ["Fluid"])) != 1:
            raise ValueError("exactly one component is supported")
        latt = js["LatticeName"][0]
        if (d, latt) not in ((2, "d2q9"), (3, "d3q19")):
            raise ValueError(f"lattice {latt} in {d}D is not supported")
        scheme = js.get("SchemeType", "Scheme_StreamCollision")
        if scheme not in abi.SCHEMES:
            raise ValueError(f"scheme {scheme} is not supported")
        sfx = "_Swap" if scheme == "Scheme_StreamCollision_Swap" else ""
        coll = js.get("CollisionType", ["Collision_BGKIsothermal2nd"])[0]
        if coll != "Collision_BGKIsothermal2nd" + sfx:
            raise ValueError(f"collision {coll} is not supported with "
                             f"{scheme}")
        force = js.get("BodyForceType", ["BodyForce_None" + sfx])[0]
        if force not in ("BodyForce_None" + sfx, "BodyForce_1st" + sfx):
            raise ValueError(f"body force {force} is not supported with "
                             f"{scheme}")
        force = force[:len(force) - len(sfx)]
        mv = js.get("MacroVarTypes", [])
        bounds = []
        i = 0
        while js.get(f"BoundaryCondition{i}") is not None:
            bc = js[f"BoundaryCondition{i}"]
            # the reference's files spell it "EQMDiffuseREfl"
            sch = bc["BoundaryScheme"]
            if sch == "EQMDiffuseREfl":
                sch = "EQMDiffuseRefl"
            bounds.append(BoundaryDef(
                block=int(bc["BlockIndex"]), surface=bc["BoundarySurface"],
                scheme=sch, vertex_type=bc["BoundaryType"],
                given=tuple(float(v) for v in bc.get("GivenVars", [])),
                macro_types=tuple(bc.get("MacroVarTypesatBoundary", []))))
            i += 1
        conns = []
        if js.get("FromBlockIds"):
            for k in range(len(js["FromBlockIds"])):
                conns.append(ConnectionDef(
                    int(js["FromBlockIds"][k]), js["FromBoundarySurface"][k],
                    int(js["ToBlockIds"][k]), js["ToBoundarySurface"][k],
                    js["BlockConnectionType"][k]))
        im = js.get("InitialMacroVars", {})
        acc = list(js.get("BodyAcceleration", [0.0, 0.0, 0.0])) + [0.0] * 3
        sp = js.get("StartPos")
        return cls(
            case_name=js.get("CaseName", "case"), space_dim=d, block_ids=ids,
            block_names=list(js.get("BlockNames", [str(v) for v in ids])),
            block_sizes=block_sizes, mesh_size=float(js["MeshSize"]),
            tau_ref=float(js["TauRef"][0]), boundaries=bounds,
            connections=conns,
            start_pos={int(k): v for k, v in sp.items()} if sp else None,
            force_velocity=any(m.endswith("_Force") for m in mv),
            body_force=force, scheme=scheme,
            accel=tuple(acc[:3]),
            initial=(float(im.get("rho", 1.0)), float(im.get("u", 0.0)),
                     float(im.get("v", 0.0)), float(im.get("w", 0.0))),
            check_period=int(js.get("CheckPeriod", 1000)),
            transient=bool(js.get("Transient", False)),
            convergence=float(js.get("ConvergenceCriteria", 1e-8)),
            steps=int(js.get("TimeStepsToRun", 0)),
            precision=js.get("Precision", "fp64"))

    @classmethod
    def load(cls, path: str) -> "CaseConfig":
        with open(path) as fh:
            return cls.from_json(json.load(fh))

    def dump(self, path: str) -> None:
        with open(path, "w") as fh:
            json.dump(self.to_json(), fh, indent=1)

    # -- C ABI descriptor ---------------------------------------------------
    def to_desc(self):
        """Returns (Desc, keepalive) for mplbgpu_create / lbmo_create."""
        nb = len(self.block_ids)
        blocks = (abi.Block * nb)()
        for i, (bid, s) in enumerate(zip(self.block_ids, self.block_sizes)):
            blocks[i].id = bid
            blocks[i].size[0] = s[0]
            blocks[i].size[1] = s[1]
            blocks[i].size[2] = s[2] if len(s) > 2 else 1
            blocks[i].cut = (self.cuts or {}).get(bid, 0)
        nc = len(self.connections)
        conns = (abi.Connection * max(nc, 1))()
        for i, c in enumerate(self.connections):
            conns[i].from_block = c.from_block
            conns[i].from_surface = abi.SURFACES[c.from_surface]
            conns[i].to_block = c.to_block
            conns[i].to_surface = abi.SURFACES[c.to_surface]
            conns[i].type = abi.VERTEX_TYPES[c.type]
        nbc = len(self.boundaries)
        bcs = (abi.Boundary * max(nbc, 1))()
        for i, b in enumerate(self.boundaries):
            bcs[i].block = b.block
            bcs[i].surface = abi.SURFACES[b.surface]
            bcs[i].scheme = abi.BC_SCHEMES[b.scheme]
            bcs[i].vertex_type = abi.VERTEX_TYPES[b.vertex_type]
            for k, v in enumerate(b.given[:3]):
                bcs[i].given[k] = v
        d = abi.Desc()
        d.abi_version = abi.ABI_VERSION
        d.space_dim = self.space_dim
        d.lattice = self.lattice
        d.precision = abi.PRECISIONS[self.precision]
        d.nblocks = nb
        d.blocks = ctypes.cast(blocks, ctypes.POINTER(abi.Block))
        d.nconnections = nc
        d.connections = ctypes.cast(conns, ctypes.POINTER(abi.Connection))
        d.nboundaries = nbc
        d.boundaries = ctypes.cast(bcs, ctypes.POINTER(abi.Boundary))
        d.tau_ref = self.tau_ref
        d.dt = self.dt
        d.cs = self.cs
        d.body_force = (abi.FORCE_1ST if self.body_force == "BodyForce_1st"
                        else abi.FORCE_NONE)
        for k in range(3):
            d.accel[k] = self.accel[k]
        d.force_velocity = 1 if self.force_velocity else 0
        d.scheme = abi.SCHEMES[self.scheme]
        return d, (blocks, conns, bcs)


# -- workload builders ------------------------------------------------------
FACES_2D = ("Left", "Right", "Top", "Bottom")
FACES_3D = ("Left", "Right", "Top", "Bottom", "Front", "Back")


def lattice_tau_to_tauref(tau_l: float, dt: float) -> float:
    """tau_L = tauRef/dt + 1/2 (Src/model_kernel.inc:428-435)."""
    return (tau_l - 0.5) * dt


def cavity(dim: int, n: int, lid_u_lattice: float, re: float = None,
           tau_lattice: float = None, wall: str = "EQMDiffuseRefl",
           order=None, precision: str = "fp64",
           check_period: int = 1000,
           scheme: str = "Scheme_StreamCollision") -> CaseConfig:
    """Lid-driven cavity with n nodes per side.  The lid is Top in 2D and
    Front (z-max) in 3D and moves along +x.  tau_L comes from Re
    (nu = U N / Re, tau = 3 nu + 1/2) unless given."""
    mesh = 1.0 / (n - 1)
    dt = mesh / SQRT3
    if tau_lattice is None:
        nu = lid_u_lattice * n / re
        tau_lattice = 3.0 * nu + 0.5
    lid_face = "Top" if dim == 2 else "Front"
    faces = list(order or (FACES_2D if dim == 2 else FACES_3D))
    lid = (SQRT3 * lid_u_lattice, 0.0, 0.0)[:dim]
    still = (0.0,) * dim
    mt = ("Variable_U", "Variable_V", "Variable_W")[:dim]
    bounds = []
    for f in faces:
        bounds.append(BoundaryDef(0, f, wall, "Wall",
                                  lid if f == lid_face else still, mt))
    return CaseConfig(
        case_name=f"cavity{dim}d", space_dim=dim, block_ids=[0],
        block_names=["Cavity"], block_sizes=[(n,) * dim], mesh_size=mesh,
        tau_ref=lattice_tau_to_tauref(tau_lattice, dt), boundaries=bounds,
        precision=precision, check_period=check_period, scheme=scheme)


def _bc(block, surface, scheme, vtype, given=(), dim=3):
    mt = {"EQMDiffuseRefl": ("Variable_U", "Variable_V", "Variable_W")[:dim],
          "HalfwayBounceBack": ("Variable_U", "Variable_V",
                                "Variable_W")[:dim],
          "ExtrapolPressure1ST": ("Variable_Rho",)}.get(scheme, ())
    return BoundaryDef(block, surface, scheme, vtype, tuple(given), mt)


def lchannel_app(n: int = 9, inflow: float = 0.001,
                 tau_ref: float = 0.01) -> CaseConfig:
    """The reference's 3D L-channel app topology (Apps/3DLChannel/
    lbm3d_L.cpp:72-205) with n nodes per side: block 0 ("Top") sits on
    block 1 ("Middle") and block 2 ("Right") to its right; block 0's Top
    wall moves with v = -inflow (inlet), block 2's Right face is a
    pressure outlet."""
    mesh = 1.0 / (n - 1)
    z0 = (0.0, 0.0, 0.0)
    mv = (0.0, -inflow, 0.0)
    bcs = [
        _bc(0, "Left", "EQMDiffuseRefl", "Wall", z0),
        _bc(0, "Right", "EQMDiffuseRefl", "Wall", z0),
        _bc(0, "Top", "EQMDiffuseRefl", "Wall", mv),
        _bc(0, "Bottom", "None", "VirtualBoundary"),
        _bc(0, "Front", "EQMDiffuseRefl", "Wall", z0),
        _bc(0, "Back", "EQMDiffuseRefl", "Wall", z0),
        _bc(1, "Left", "EQMDiffuseRefl", "Wall", z0),
        _bc(1, "Right", "None", "VirtualBoundary"),
        _bc(1, "Top", "None", "VirtualBoundary"),
        _bc(1, "RightTop", "EQMDiffuseRefl", "Wall", z0),
        _bc(1, "Bottom", "EQMDiffuseRefl", "Wall", z0),
        _bc(1, "Front", "EQMDiffuseRefl", "Wall", z0),
        _bc(1, "Back", "EQMDiffuseRefl", "Wall", z0),
        _bc(2, "Left", "None", "VirtualBoundary"),
        _bc(2, "Right", "ExtrapolPressure1ST", "OutLet", (1.0,)),
        _bc(2, "Top", "EQMDiffuseRefl", "Wall", z0),
        _bc(2, "Bottom", "EQMDiffuseRefl", "Wall", z0),
        _bc(2, "Front", "EQMDiffuseRefl", "Wall", z0),
        _bc(2, "Back", "EQMDiffuseRefl", "Wall", z0),
    ]
    conns = [ConnectionDef(0, "Bottom", 1, "Top", "VirtualBoundary"),
             ConnectionDef(1, "Top", 0, "Bottom", "VirtualBoundary"),
             ConnectionDef(1, "Right", 2, "Left", "VirtualBoundary"),
             ConnectionDef(2, "Left", 1, "Right", "VirtualBoundary")]
    return CaseConfig(
        case_name="lchannel_app", space_dim=3, block_ids=[0, 1, 2],
        block_names=["Top", "Middle", "Right"],
        block_sizes=[(n, n - 1, n), (n, n, n), (n - 1, n, n)],
        mesh_size=mesh, tau_ref=tau_ref, boundaries=bcs, connections=conns)


def lchannel(leg: int = 384, side: int = 128, depth: int = 128,
             inlet_u_lattice: float = 0.03, tau_lattice: float = 0.6,
             wall: str = "EQMDiffuseRefl", precision: str = "fp64",
             check_period: int = 1000) -> CaseConfig:
    """3D L-shaped channel of three blocks joined on one GPU: block 0 is the
    inlet leg (leg x side x depth, inlet on its Left face), block 1 the
    corner (side x side x depth), block 2 the outlet leg (side x leg x
    depth, pressure outlet rho = 1 on its Top face).  z is periodic on every
    block (MDPeriodic self-connections); the other faces are walls."""
    mesh = 1.0 / (side - 1)
    dt = mesh / SQRT3
    z0 = (0.0, 0.0, 0.0)
    inlet = (SQRT3 * inlet_u_lattice, 0.0, 0.0)
    wt = "Fluid" if wall == "HalfwayBounceBack" else "Wall"
    bcs = []
    for b in (0, 1, 2):
        bcs += [_bc(b, "Front", "MDPeriodic", "MDPeriodic"),
                _bc(b, "Back", "MDPeriodic", "MDPeriodic")]
    bcs += [
        _bc(0, "Top", wall, wt, z0), _bc(0, "Bottom", wall, wt, z0),
        _bc(0, "Left", "EQMDiffuseRefl", "Inlet", inlet),
        _bc(0, "Right", "None", "VirtualBoundary"),
        _bc(1, "Right", wall, wt, z0), _bc(1, "Bottom", wall, wt, z0),
        _bc(1, "Left", "None", "VirtualBoundary"),
        _bc(1, "Top", "None", "VirtualBoundary"),
        _bc(1, "LeftTop", wall, wt, z0),
        _bc(2, "Left", wall, wt, z0), _bc(2, "Right", wall, wt, z0),
        _bc(2, "Bottom", "None", "VirtualBoundary"),
        _bc(2, "Top", "ExtrapolPressure1ST", "OutLet", (1.0,)),
    ]
    conns = [ConnectionDef(0, "Right", 1, "Left", "VirtualBoundary"),
             ConnectionDef(1, "Left", 0, "Right", "VirtualBoundary"),
             ConnectionDef(1, "Top", 2, "Bottom", "VirtualBoundary"),
             ConnectionDef(2, "Bottom", 1, "Top", "VirtualBoundary")]
    for b in (0, 1, 2):
        conns += [ConnectionDef(b, "Front", b, "Back", "MDPeriodic"),
                  ConnectionDef(b, "Back", b, "Front", "MDPeriodic")]
    return CaseConfig(
        case_name="lchannel", space_dim=3, block_ids=[0, 1, 2],
        block_names=["InletLeg", "Corner", "OutletLeg"],
        block_sizes=[(leg, side, depth), (side, side, depth),
                     (side, leg, depth)],
        mesh_size=mesh, tau_ref=lattice_tau_to_tauref(tau_lattice, dt),
        boundaries=bcs, connections=conns, precision=precision,
        check_period=check_period)


def inlet_index(case: CaseConfig) -> int:
    """Position in the boundary list (definition order) of the case's one
    boundary with vertex type Inlet."""
    idx = [k for k, b in enumerate(case.boundaries) if b.vertex_type == "Inlet"]
    if len(idx) != 1:
        raise ValueError("the case has no single Inlet boundary")
    return idx[0]


def face_extent(case: CaseConfig, k: int) -> Tuple[int, int, int]:
    """(nx, ny, nz) of the node range of face boundary k (Left/Right: one
    x layer, Bottom/Top: one y layer, Back/Front: one z layer)."""
    bc = case.boundaries[k]
    nx, ny, nz = case.size3(bc.block)
    axis = {"Left": 0, "Right": 0, "Bottom": 1, "Top": 1, "Back": 2,
            "Front": 2}.get(bc.surface)
    if axis is None:
        raise ValueError(f"boundary {k} is not a face")
    ext = [nx, ny, nz]
    ext[axis] = 1
    return tuple(ext)


def inlet_perturbation(case: CaseConfig, seed: int = 20261203,
                       amplitude: float = 0.01):
    """Per-node inlet velocity (MPLB units) for the case's Inlet face: the
    boundary's given velocity with its normal component scaled by
    1 + e, e uniform in [-amplitude, amplitude] per node, drawn from
    numpy's PCG64 generator seeded with `seed` in node order (x fastest,
    then y, then z).  Returns (boundary index, (u, v, w)) with arrays of
    shape (nz, ny, nx) over the face.  The reference takes one uniform
    velocity per boundary (GivenVars), so this is an extension of it."""
    import numpy as np
    k = inlet_index(case)
    nx, ny, nz = face_extent(case, k)
    bc = case.boundaries[k]
    g = list(bc.given) + [0.0] * (3 - len(bc.given))
    axis = {"Left": 0, "Right": 0, "Bottom": 1, "Top": 1, "Back": 2,
            "Front": 2}[bc.surface]
    e = np.random.default_rng(seed).uniform(-amplitude, amplitude,
                                            size=(nz, ny, nx))
    comps = [np.full((nz, ny, nx), g[a]) for a in range(3)]
    comps[axis] = g[axis] * (1.0 + e)
    if case.space_dim == 2:
        comps[2] = None
    return k, tuple(comps)


def poiseuille(dim: int, nx: int, ny: int, nz: int = 1,
               g_lattice: float = 1e-6, tau_lattice: float = 0.8,
               wall: str = "EQMDiffuseRefl", precision: str = "fp64",
               check_period: int = 1000) -> CaseConfig:
    """Body-force driven channel: walls at y-min/y-max, periodic in x (and
    z) through MDPeriodic self-connections, force along +x with the
    force-corrected velocity moments (Variable_U_Force family).  The
    lattice acceleration g_L is a_MPLB = g_L dx / dt^2 in MPLB units."""
    ny_mesh = ny - 1 if wall != "HalfwayBounceBack" else ny
    mesh = 1.0 / ny_mesh
    dt = mesh / SQRT3
    a = g_lattice * mesh / (dt * dt)
    wt = "Fluid" if wall == "HalfwayBounceBack" else "Wall"
    z0 = (0.0,) * dim
    bcs = [_bc(0, "Left", "MDPeriodic", "MDPeriodic", dim=dim),
           _bc(0, "Right", "MDPeriodic", "MDPeriodic", dim=dim)]
    conns = [ConnectionDef(0, "Left", 0, "Right", "MDPeriodic"),
             ConnectionDef(0, "Right", 0, "Left", "MDPeriodic")]
    if dim == 3:
        bcs += [_bc(0, "Front", "MDPeriodic", "MDPeriodic"),
                _bc(0, "Back", "MDPeriodic", "MDPeriodic")]
        conns += [ConnectionDef(0, "Front", 0, "Back", "MDPeriodic"),
                  ConnectionDef(0, "Back", 0, "Front", "MDPeriodic")]
    bcs += [_bc(0, "Top", wall, wt, z0, dim), _bc(0, "Bottom", wall, wt, z0,
                                                   dim)]
    size = (nx, ny) if dim == 2 else (nx, ny, nz)
    return CaseConfig(
        case_name=f"poiseuille{dim}d", space_dim=dim, block_ids=[0],
        block_names=["Channel"], block_sizes=[size], mesh_size=mesh,
        tau_ref=lattice_tau_to_tauref(tau_lattice, dt), boundaries=bcs,
        connections=conns, force_velocity=True, body_force="BodyForce_1st",
        accel=(a, 0.0, 0.0), precision=precision, check_period=check_period)
