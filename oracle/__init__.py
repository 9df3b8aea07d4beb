"""CPU oracle for the PRT-LB hot path -- TEST INFRASTRUCTURE ONLY.

A NumPy restatement of the reference's algorithms (shahram444/PRT-DeepONet-GUI,
3D/tools/prtlb_2d.py and 3D/tools/prtlb_3d.py), used to check the CUDA path:

    prtlb_oracle.stokes        the D2Q9 / D3Q19 TRT flow solve, float64
    prtlb_oracle.solve_adr     the transport solve, float32 (the reference's
                               precision) or float64 (its float64 twin)
    pairwise.pairwise_sum      numpy's float32 pairwise summation order

Parity is pinned: tests/test_oracle_golden.py checks these functions against
golden vectors produced by the reference itself (tests/golden/make_golden.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker or the timed CPU baseline; the
product (prt-deeponet-gui_b200/prtlb_gpu) never does.
"""
