"""Descriptor files e%06d in the layout the reference's parse step writes
(LNK_OUT, src/nprs.c:380-442) and its training reads (LNK_IN,
src/nprs.c:308-377):

    EFS D N NF DNn E p DE
    [EFS 1, 3]  indices of the marked atoms
    [EFS 2, 3]  the six reference stresses
    data path
    per atom: species, then D descriptors
    [EFS 1, 3]  per marked atom, in atom order: i DNn F_x F_y F_z, the D rows
                of the self block dG_i/dx_i, then DNn times: owner index j and
                the D rows of dG_j/dx_i
    [EFS 2, 3]  per atom the D rows of dG/dstrain (6 values)

Read token by token, as LNK_IN's fscanf does.  mb_parse_efile
(Potential.parse_efile) writes the same layout.
"""
from __future__ import annotations

import os

import numpy as np


def read_efile(directory, index):
    """dict(EFS, D, N, NF, E, p, DE, path, atmn[N], G[N, D], marked[NF],
    F[NF, 3], blocks: list of (atom, owners[DNn + 1], Fn[DNn + 1, D, 3]) with
    the self block last and owner = atom, S[6], Sn[N, D, 6])."""
    with open(os.path.join(directory, f"e{index:06d}")) as f:
        tok = f.read().split()
    pos = 0

    def take(k):
        nonlocal pos
        out = tok[pos:pos + k]
        if len(out) < k:
            raise ValueError(f"descriptor file e{index:06d} ends early")
        pos += k
        return out

    EFS, D, N, NF, DNn = (int(v) for v in take(5))
    E, p, DE = (float(v) for v in take(3))
    out = dict(EFS=EFS, D=D, N=N, NF=NF, DNn=DNn, E=E, p=p, DE=DE)
    marked = np.array([int(v) for v in take(NF)], np.int32) if EFS in (1, 3) else np.zeros(0, np.int32)
    if EFS in (2, 3):
        out["S"] = np.array([float(v) for v in take(6)])
    out["path"] = take(1)[0]
    atmn = np.zeros(N, np.int32)
    G = np.zeros((N, D))
    for i in range(N):
        atmn[i] = int(take(1)[0])
        G[i] = np.array(take(D), float)
    out["atmn"], out["G"] = atmn, G
    blocks, F = [], np.zeros((NF, 3))
    if EFS in (1, 3):
        order = {int(a): k for k, a in enumerate(sorted(set(marked.tolist())))}
        for _ in range(len(order)):
            atom, dnn = int(take(1)[0]), int(take(1)[0])
            f = np.array(take(3), float)
            Fn = np.zeros((dnn + 1, D, 3))
            Fn[dnn] = np.array(take(3 * D), float).reshape(D, 3)
            owners = np.zeros(dnn + 1, np.int32)
            for j in range(dnn):
                owners[j] = int(take(1)[0])
                Fn[j] = np.array(take(3 * D), float).reshape(D, 3)
            owners[dnn] = atom
            blocks.append((atom, owners, Fn))
            F[order[atom]] = f
    out["marked"], out["blocks"] = np.array(sorted(set(marked.tolist())), np.int32), blocks
    out["F"] = F[:len(blocks)]
    if EFS in (2, 3):
        out["Sn"] = np.array(take(N * D * 6), float).reshape(N, D, 6)
    return out
