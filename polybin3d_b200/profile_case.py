"""Small single-kernel case for profiling: one bispectrum numerator (filter, c2r, triplet
contraction) of a seeded lognormal field, nothing else.

    python -m polybin3d_b200.profile_case [N] [L] [kmax] [nk] [lmax] [contraction]
"""
import contextlib
import io
import sys

import numpy as np
import torch


def main(argv):
    import polybin3d_b200 as pb
    from polybin3d_b200 import synthetic
    N = int(argv[0]) if len(argv) > 0 else 256
    L = float(argv[1]) if len(argv) > 1 else 2000.0
    kmax = float(argv[2]) if len(argv) > 2 else 0.2
    nk = int(argv[3]) if len(argv) > 3 else 16
    lmax = int(argv[4]) if len(argv) > 4 else 2
    contraction = argv[5] if len(argv) > 5 else "simt"
    with contextlib.redirect_stdout(io.StringIO()):
        base = pb.PolyBin3D([L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
        bs = pb.BSpec(base, np.linspace(2 * np.pi / L, kmax, nk + 1), lmax=lmax, contraction=contraction)
    bs.sym_factor = np.ones(bs.N_bins)
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=0), device=base.device)
    for _ in range(2):
        out = bs._bk_cubic(d, "ideal")
    torch.cuda.synchronize()
    print("ok", bs.map_grid, float(out.abs().max()))


if __name__ == "__main__":
    main(sys.argv[1:])
