"""Splitting a domain into MeshBlocks along x2 / x3 (host logic only).

A domain Problem (one block's configuration and state) is cut into
nb2 x nb3 equal blocks, as Athena's Mesh cuts its root grid into MeshBlocks
(`<meshblock>` nx2 / nx3).  x1, the vertical, is never cut: the hydrostatic
scan and the implicit column solve stay inside a block.  Sides between
blocks, and the domain's periodic sides when the direction has more than one
block, become CANOE_BC_BLOCK sides whose neighbour is the adjoining block
(Athena's periodic neighbour wraps around the root grid the same way).

Block (b2, b3) has index b3 * nb2 + b2.  `neighbors` lists, per block and
per side 2..5 (ix2, ox2, ix3, ox3), the index of the neighbour or None.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._abi import BC_BLOCK, BC_PERIODIC, NGHOST, BlockConfig


@dataclass
class Split:
    nb2: int
    nb3: int
    blocks: list            # Problem per block
    offsets: list           # (o2, o3): first interior cell of the block in the domain
    neighbors: list = field(default_factory=list)  # per block: {side: index}


def _copy_cfg(cfg):
    c = BlockConfig()
    ctypes.memmove(ctypes.addressof(c), ctypes.addressof(cfg), ctypes.sizeof(BlockConfig))
    return c


def _interior_slices(cfg):
    ng = NGHOST
    ks = ng if cfg.nx3 > 1 else 0
    js = ng if cfg.nx2 > 1 else 0
    return slice(ks, ks + cfg.nx3), slice(js, js + cfg.nx2)


def split(problem, nb2, nb3=1):
    """Cut `problem` into nb2 x nb3 blocks (each direction's cell count must
    divide evenly, with at least NGHOST cells per block where cut)."""
    from .problems import Problem, _shape
    cfg = problem.cfg
    if nb2 < 1 or nb3 < 1 or cfg.nx2 % nb2 or cfg.nx3 % nb3:
        raise ValueError("the block counts must divide nx2 and nx3")
    if (nb2 > 1 and cfg.nx2 // nb2 < NGHOST) or (nb3 > 1 and cfg.nx3 // nb3 < NGHOST):
        raise ValueError("a block needs at least NGHOST cells along a cut direction")
    if (nb2 > 1 and cfg.nx2 == 1) or (nb3 > 1 and cfg.nx3 == 1):
        raise ValueError("cannot cut a direction without cells")
    n2, n3 = cfg.nx2 // nb2, cfg.nx3 // nb3
    k_dom, j_dom = _interior_slices(cfg)
    out = Split(nb2, nb3, [], [])
    for b3 in range(nb3):
        for b2 in range(nb2):
            c = _copy_cfg(cfg)
            c.nx2, c.nx3 = n2, n3
            c.x2min = cfg.x2min + b2 * n2 * cfg.dx2
            c.x3min = cfg.x3min + b3 * n3 * cfg.dx3
            nbr = {}
            for side, (nb, b, cnt, lo_side) in {
                    2: (nb2, b2, nb2, True), 3: (nb2, b2, nb2, False),
                    4: (nb3, b3, nb3, True), 5: (nb3, b3, nb3, False)}.items():
                if nb == 1:
                    continue  # the domain's own boundary condition stays
                edge = (b == 0) if lo_side else (b == cnt - 1)
                if edge and cfg.bc[side] != BC_PERIODIC:
                    continue  # a physical wall of the domain
                c.bc[side] = BC_BLOCK
                step = -1 if lo_side else 1
                if side < 4:
                    nbr[side] = b3 * nb2 + (b2 + step) % nb2
                else:
                    nbr[side] = ((b3 + step) % nb3) * nb2 + b2
            c.h_x1f = cfg.h_x1f
            shape = _shape(cfg.nx1, n2, n3, problem.nv)
            u = np.zeros(shape)
            kb, jb = _interior_slices(c)
            o2, o3 = b2 * n2, b3 * n3
            u[:, kb, jb, :] = problem.u[:, k_dom.start + o3:k_dom.start + o3 + n3,
                                        j_dom.start + o2:j_dom.start + o2 + n2, :]
            p = Problem(f"{problem.name}[{b2},{b3}]", c, problem.x1f, u, np.zeros(shape),
                        dict(problem.meta))
            out.blocks.append(p)
            out.offsets.append((o2, o3))
            out.neighbors.append(nbr)
    return out


def gather(sp, domain_shape, states, nx2, nx3):
    """Assemble the blocks' arrays (NV, nc3b, nc2b, nc1) into a domain array
    of domain_shape (interior cells; the domain's ghosts stay zero)."""
    out = np.zeros(domain_shape)
    ks = NGHOST if nx3 > 1 else 0
    js = NGHOST if nx2 > 1 else 0
    for p, (o2, o3), a in zip(sp.blocks, sp.offsets, states):
        kb, jb = _interior_slices(p.cfg)
        n3, n2 = p.cfg.nx3, p.cfg.nx2
        out[:, ks + o3:ks + o3 + n3, js + o2:js + o2 + n2, :] = a[:, kb, jb, :]
    return out
