"""The inflow fill of the USERDEF parity cases, on the device.

The same rule as UserDefBoundary in oracle/ref/init.cpp (the problem file
the reference fixtures were made with) and the oracle's USERDEF branch:
every ghost cell of the side takes the primitive state of the domain cell
next to the side, then density UD_RHO and the normal velocity UD_VN into the
domain; the tangential face fields copy the domain face next to the side
over the whole extent of the other directions.  It runs as torch copies on
the library's stream through the USERDEF callback of the C ABI.
"""
import oracle as orc
from gpluto_dev_b200 import ics

UD_RHO, UD_VN = orc.UD_RHO, orc.UD_VN


def inflow_fill(side):
    V, Vs = side.tensors()
    d = side.side // 2
    beg = side.side % 2 == 0
    m0 = side.dom_beg[d] if beg else side.dom_beg[d] + side.nint[d] - 1
    g0, ng = side.beg[d], side.end[d] - side.beg[d] + 1
    with side.torch_stream():
        ax = 3 - d                      # V is [nvar, z, y, x]
        dst = V.narrow(ax, g0, ng)
        dst.copy_(V.narrow(ax, m0, 1).expand_as(dst))
        dst[ics.RHO] = UD_RHO
        dst[ics.VX1 + d] = UD_VN if beg else -UD_VN
        for e, B in enumerate(Vs):
            if B is None or e == d:
                continue
            bx = 2 - d                  # face fields are [z, y, x]
            bd = B.narrow(bx, g0, ng)
            bd.copy_(B.narrow(bx, m0, 1).expand_as(bd))
