"""Child process of test_gpu_builders.py: computes tensor-core fields (single
fields in both CTA forms, and one batch) with whatever table-builder form the
environment selects, and saves them to the .npz file named on the command
line. The builder form is read once per process, hence the child."""
import ctypes
import sys
from pathlib import Path

import numpy as np
import torch

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
sys.path.insert(0, str(Path(__file__).resolve().parent))
import scarf3d_b200 as sb  # noqa: E402
from srm_cases import iarr, structured_case  # noqa: E402

CASES = ["vk3d", "gs3d_aniso", "vk3d_rot_offset", "gs2d"]
BATCH = [(48, 32, 64), (80, 16, 32), (17, 23, 40), (64, 64, 128)]


def single(name, variant):
    c = structured_case(name)
    s = sb.compute_setup(c["pp"])
    tab, _ = sb.sample(c["pp"], s)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    n = c["n"]
    out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    sb.set_tc_variant(variant)
    wb = sb.tc_workspace_bytes(c["nd"], n, len(tab))
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(c["fs"]), iarr(n), c["ds"],
                                            ctypes.c_void_p(d_tab.data_ptr()), len(tab),
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                            wb, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def batch():
    entries, outs, keep = [], [], []
    for f, n in enumerate(BATCH):
        cl = [float(min(2000.0, max(300.0, (m - 1) * 50.0 / 3.5))) for m in n]
        fc = [float(np.float32(m - 1) * np.float32(50.0)) for m in n]
        p = sb.make_params(nc=[0.0] * 3, fc=fc, acf=f % 2, nharm=200 + 50 * f, seed=70 + f,
                           hurst=0.3 if f % 2 == 0 else 0.0, sigma=0.05, ds=50.0, cl=cl)
        s = sb.compute_setup(p)
        tab, _ = sb.sample(p, s)
        d = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
        o = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
        keep.append(d)
        outs.append(o)
        entries.append(dict(setup=s, fs=[1, 1, 1], n=list(n), ds=50.0, d_table=d.data_ptr(), nh=len(tab),
                            d_field=o.data_ptr()))
    b = sb.TcBatch(entries, lambda nb: torch.empty(nb, dtype=torch.uint8, device="cuda"))
    b.launch()
    b.wait()
    return [o.cpu().numpy() for o in outs]


def main(path):
    res = {}
    for name in CASES:
        for variant, tag in ((sb.TC_SINGLE, "single"), (sb.TC_PAIR, "pair")):
            res[f"{name}_{tag}"] = single(name, variant)
    sb.set_tc_variant(sb.TC_SINGLE)
    for f, o in enumerate(batch()):
        res[f"batch{f}"] = o
    np.savez(path, **res)


if __name__ == "__main__":
    main(sys.argv[1])
