"""Cases shared by several tests that are neither golden fixtures nor
seeded random cases."""
import dataclasses

from mplb_b200 import config


def fdperiodic_channel():
    """A forced channel made x-periodic through FDPeriodic boundaries and
    connections (the reference's KerCutCellPeriodic3D path, whose copies
    read a halo of f that no step writes)."""
    c = config.poiseuille(3, 8, 7, 6, g_lattice=1e-4)
    bcs = [dataclasses.replace(b, scheme="FDPeriodic",
                               vertex_type="FDPeriodic")
           if b.surface in ("Left", "Right") else b for b in c.boundaries]
    conns = [dataclasses.replace(x, type="FDPeriodic")
             if x.from_surface in ("Left", "Right") else x
             for x in c.connections]
    return dataclasses.replace(c, boundaries=bcs, connections=conns)


def fdperiodic_box(dim=3):
    """A cavity whose faces mix FDPeriodic and EQMDiffuseRefl in an order
    that sends the edge and corner nodes through the reference's edge and
    corner cases of KerCutCellPeriodic(3D) (the mislabelled ones
    included)."""
    c = config.cavity(dim, 7, 0.05, re=100)
    fd = {"Left", "Front", "Right", "Bottom"}
    order = (["Top", "Left", "Front", "Right", "Back", "Bottom"] if dim == 3
             else ["Top", "Left", "Right", "Bottom"])
    by = {b.surface: b for b in c.boundaries}
    bcs = []
    for s in order:
        b = by[s]
        if s in fd:
            b = dataclasses.replace(b, scheme="FDPeriodic",
                                    vertex_type="FDPeriodic")
        bcs.append(b)
    return dataclasses.replace(c, boundaries=bcs)
