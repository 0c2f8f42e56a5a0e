"""The reference's own CUDA PP kernel beside this build's, on one GPU -- a
measurement script (it loads oracle/_ref/, so it lives with the tests).

The reference's updateKernel (lcl_g_2.cu:7-103, launched through the harness
oracle/ref_pp_cuda.cu with the reference's launch shape) is hard-wired to
r_c = 3 (37 slots per cell). At that cutoff, on seeded uniform positions at
the reference's number density 3/(4 pi), this times

* updateKernel (linked cells, one thread per particle, FP32/FP64 mix);
* this build's FP32 pair kernel over its Verlet lists (and, apart, one full
  list rebuild), through a PP-only context (no mesh);

and checks both against the oracle's FP64 PP (yukawa_pp.py:6-139 restated).

    python tests/ref_cuda_pp_report.py [N]
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "md-force-routines_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

LIB = os.path.join(ROOT, "oracle", "_ref", "libref_pp_cuda.so")


def main(argv):
    import initialize_pos_vel
    from oracle import oracle as O
    from p3m_b200 import FP32, Context, Replica

    N = int(argv[0]) if argv else 200000
    kappa, alpha, rc = 2.0, 0.6, 3.0
    L = (4 * np.pi * N / 3) ** (1 / 3)
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(11, N, [L] * 3, pos, vel, 0.01)
    pos = np.where(pos >= L, pos - L, pos)
    U_o, a_o = O.pp(kappa, alpha, rc, [L] * 3, pos)
    out = {"N": N, "L": L, "kappa": kappa, "alpha": alpha, "rc": rc}

    lib = ctypes.CDLL(LIB)
    fp = ctypes.POINTER(ctypes.c_float)
    lib.ref_update_kernel.argtypes = [ctypes.c_int, fp, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_int, fp, fp]
    p32 = np.ascontiguousarray(pos, dtype=np.float32)
    acc_r = np.zeros((N, 3), dtype=np.float32)
    ms = np.zeros(1, dtype=np.float32)
    rcode = lib.ref_update_kernel(N, p32.ctypes.data_as(fp), L, kappa, alpha, rc, 20,
                                  acc_r.ctypes.data_as(fp), ms.ctypes.data_as(fp))
    assert rcode == 0, rcode

    def err(a):
        return float(np.sqrt(np.sum((a - a_o) ** 2) / np.sum(a_o ** 2)))

    out["reference_updateKernel"] = {"ms_per_launch": float(ms[0]),
                                     "rms_err_vs_oracle": err(acc_r.astype(np.float64)),
                                     "launch": "grid (512, ceil(Ncell/512)), 64 threads"}
    rep = Replica(N=N, L=L, kappa=kappa, alpha=alpha, rc=rc, M=0)
    with Context(rep, precision=FP32) as c:
        U, a = c.pp(pos)
        c.set_state(0, pos, vel)
        c.init_forces()
        st = c.profile_stages(iters=50)
        tpi, skin, _ = c.pp_config()
    out["this_build_fp32"] = {"pp_kernel_ms": st.get("pp"), "list_rebuild_ms": st.get("keys_sort"),
                              "threads_per_particle": tpi, "skin": skin,
                              "rms_err_vs_oracle": err(a), "U_rel_err": abs(U - U_o) / abs(U_o)}
    print(json.dumps(out))


if __name__ == "__main__":
    main(sys.argv[1:])
