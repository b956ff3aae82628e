"""The 'auto' choice between the direct solver and AMG-PCG (autoSolverChoice, physics/src/common/scalar.ts:264-283):
the reference's rule and messages with its CPU thresholds, and the same rule with this GPU factor's thresholds."""
import ampsolve as amp
import workloads as wl

CPU = {"flopsPerDof": amp.AUTO_FLOPS_PER_DOF_CPU, "maxFactorBytes": amp.AUTO_MAX_FACTOR_BYTES_CPU}


def test_reference_rule_and_messages():
    # the two measured points of the reference's break-even note: 2.7e5 flop/DOF (direct) and 7.6e5 (AMG-PCG)
    assert amp.autoSolverChoice(15600, 2.7e5 * 15600, 10 ** 6, **CPU) == \
        {"kind": "cholesky", "reason": "direct factor 2.70e+5 flop/DOF < 3e+5"}
    assert amp.autoSolverChoice(35900, 7.6e5 * 35900, 10 ** 6, **CPU) == \
        {"kind": "amg-pcg", "reason": "direct factor 7.60e+5 flop/DOF >= 3e+5"}
    # the break-even itself goes to AMG-PCG (>=); 2D tri6 at 4.0e4 stays direct
    assert amp.autoSolverChoice(1000, 3e8, 10, **CPU)["kind"] == "amg-pcg"
    assert amp.autoSolverChoice(646000, 4.0e4 * 646000, 10 ** 7, **CPU)["reason"] == "direct factor 4.00e+4 flop/DOF < 3e+5"
    # memory first: 8 nnzL bytes above 1 GiB, whatever the flop count
    assert amp.autoSolverChoice(10, 1.0, 2 ** 27 + 1, **CPU) == \
        {"kind": "amg-pcg", "reason": "direct factor 1024 MiB > 1024 MiB"}
    assert amp.autoSolverChoice(10, 1.0, 3 * 2 ** 27, **CPU)["reason"] == "direct factor 3072 MiB > 1024 MiB"


def test_number_formatting_rounds_half_up():
    assert amp._js_exp(266500.0, 2) == "2.67e+5"  # toExponential rounds the exact value half up (not to even)
    assert amp._js_exp(999500.0, 2) == "1.00e+6"
    assert amp._js_exp(3e5, 0) == "3e+5" and amp._js_exp(1.7e8, 0) == "2e+8"
    assert amp._js_fixed0(2.5) == "3" and amp._js_fixed0(1024.0) == "1024"


def test_gpu_thresholds_keep_3d_systems_direct():
    # 3D elasticity 40^3: 0.79 TFLOP over 201,720 DOF = 3.9e6 flop/DOF, AMG-PCG by the CPU rule, direct on the GPU
    n, flops, nnzl = 201720, 0.79e12, 2.0e8
    assert amp.autoSolverChoice(n, flops, nnzl, **CPU)["kind"] == "amg-pcg"
    assert amp.autoSolverChoice(n, flops, nnzl)["kind"] == "cholesky"
    # beyond the device memory budget: AMG-PCG
    assert amp.autoSolverChoice(n, flops, nnzl, factorBytes=200 * 2 ** 30)["kind"] == "amg-pcg"
    sym = amp.analyze(wl.elastic3d(8).pat)
    c = amp.autoSolverChoiceFor(sym)
    assert c["kind"] == "cholesky" and sym.deviceBytes > 0
