"""Algorithmic work per element of the elemental step, used for the roofline report.

The counts follow the reference's operation sequence (the dense-BLAS forms of
kernel/volint.m, kernel/faceint.m and kernel/schur_uq.c), not the cheaper sum-factorised
forms the kernel executes, so a kernel that skips work reads as faster, not as more FLOPs:

  schur   = npv^3/3 + 2 npv^2 nd (ncu+npv+ndf) + 2 nu npv ncu nd + 2 nd ncu nu npv (npv+ndf)
            + 2/3 nu^3 + 2 nu^2 (1+nh) + 2 nd npv^2 ncu (1+nh) + 2 nh^2 nuq + 2 nh nuq
  assembly = 2 npv^2 ngv (nd+1) ncu nc + 2 npv^2 ngv (1+nd^2) + 4 npf^2 ngf nfe ncu (nc+ncu)
  bytes   = 8 * (dgnodes + UDG + UH + SH + AE + FE + DUDG + DUDG_DUH) + 4 * bf
with nu = npv ncu, nuq = npv nc, nh = ncu ndf, ndf = npf nfe.
"""
from __future__ import annotations


def element_counts(nd, npv, npf, ngv, ngf, ncu=None):
    ncu = nd + 2 if ncu is None else ncu
    nc = ncu * (nd + 1)
    nfe = nd + 1
    ndf = npf * nfe
    nu, nuq, nh = npv * ncu, npv * nc, ncu * ndf
    schur = (npv ** 3 / 3 + 2 * npv ** 2 * nd * (ncu + npv + ndf) + 2 * nu * npv * ncu * nd
             + 2 * nd * ncu * nu * npv * (npv + ndf) + 2.0 / 3.0 * nu ** 3 + 2 * nu ** 2 * (1 + nh)
             + 2 * nd * npv ** 2 * ncu * (1 + nh) + 2 * nh ** 2 * nuq + 2 * nh * nuq)
    assembly = (2 * npv ** 2 * ngv * (nd + 1) * ncu * nc + 2 * npv ** 2 * ngv * (1 + nd ** 2)
                + 4 * npf ** 2 * ngf * nfe * ncu * (nc + ncu))
    bytes_in = 8 * (npv * nd + npv * nc + ncu * ndf + npv * nc) + 4 * nfe
    bytes_out = 8 * (nh * nh + nh + nuq + nuq * nh)
    return dict(schur_flops=schur, assembly_flops=assembly, flops=schur + assembly,
                bytes_in=bytes_in, bytes_out=bytes_out, bytes=bytes_in + bytes_out)
