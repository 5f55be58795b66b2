#!/usr/bin/env python3
"""TEST INFRASTRUCTURE ONLY: copies the reference's QuantumSimEvo sources into a
build directory (oracle/_ref/patched: git-ignored, never the repository, never
the reference tree) and patches two of them there, so the reference's own
Circuit can be compiled with the optional backend hooks that hand a whole gate
queue and the sampling draws to the backend.  The whole directory is copied so
that every translation unit, including the reference headers that include the
interface from their own directory, sees the same patched interface.

  python oracle/patch_reference.py <reference QuantumSimEvo dir> <output dir>

The edits are the ones a maintainer adopting the B200 backend would make:

ICircuitUnitaryOperation.h (ICircuitUnitaryOperation.h:6-35): three virtuals
with defaults that decline (return false), so the scalar, AVX2 and CUDA
backends are untouched:
    virtual bool executeProgram(StateVector&, const std::vector<GateCommand>&);
    virtual bool sample(StateVector&, const double* u, size_t shots, std::vector<size_t>& out);
    virtual bool measure(StateVector&, double u, size_t& out);

Circuit.cpp (Circuit.cpp:64-143):
  - Circuit::execute offers the whole queue to executeProgram first when noise
    is off and print_steps is false, and keeps its per-gate loop otherwise;
  - Circuit::sample / Circuit::measure draw their uniforms in [0, 1) and offer
    them to the backend before falling back to flush() + the host StateVector.
    The draws come from qse_patch_next_uniform(), which the test shim defines
    (injected values for parity tests, a random_device-seeded generator
    otherwise, like the reference's own std::random_device draws).

Every anchor is checked; the script fails if the reference text differs.
"""
import os
import re
import shutil
import sys

HOOKS = """
    // Optional whole-program and device-sampling hooks.  The defaults decline
    // (return false) and the caller keeps its per-gate loop / host sampling.
    virtual bool executeProgram(StateVector& sv, const std::vector<GateCommand>& commands)
    { (void)sv; (void)commands; return false; }
    virtual bool sample(StateVector& sv, const double* u, size_t shots, std::vector<size_t>& out)
    { (void)sv; (void)u; (void)shots; (void)out; return false; }
    virtual bool measure(StateVector& sv, double u, size_t& out)
    { (void)sv; (void)u; (void)out; return false; }
"""

EXEC_HOOK = """
    if (!simulateNoise && !print_steps && circuitOp->executeProgram(stateVector, commands))
        return;
"""

MEASURE_HOOK = """
    {
        size_t out = 0;
        if (circuitOp->measure(stateVector, qse_patch_next_uniform(), out)) return out;
    }
"""

SAMPLE_HOOK = """
    {
        std::vector<double> u(numShots > 0 ? size_t(numShots) : 0);
        for (double& x : u) x = qse_patch_next_uniform();
        std::vector<size_t> out;
        if (circuitOp->sample(stateVector, u.data(), u.size(), out)) return out;
    }
"""


def patch_once(text, pattern, repl, what):
    new, count = re.subn(pattern, repl, text, count=1, flags=re.S)
    if count != 1:
        raise SystemExit(f"patch_reference: anchor not found for {what}")
    return new


def main():
    src, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    for name in os.listdir(src):
        if name.endswith((".h", ".cpp", ".cu")):
            shutil.copyfile(os.path.join(src, name), os.path.join(out, name))
    with open(os.path.join(src, "ICircuitUnitaryOperation.h")) as f:
        h = f.read()
    h = patch_once(h, r'(#include "StateVector.h"\n)', r'\1#include "Structurs.h"\n', "interface includes")
    h = patch_once(h, r"(virtual void markHostDirty\(\) \{\}\n)", lambda m: m.group(1) + HOOKS, "interface hooks")
    with open(os.path.join(out, "ICircuitUnitaryOperation.h"), "w") as f:
        f.write(h)

    with open(os.path.join(src, "Circuit.cpp")) as f:
        c = f.read()
    c = "// test hook: the draw source of Circuit::sample / measure (defined by the test shim)\n" \
        "double qse_patch_next_uniform();\n" + c
    c = patch_once(c, r"(void Circuit::execute\(bool print_steps\) \{\n)", lambda m: m.group(1) + EXEC_HOOK,
                   "Circuit::execute")
    c = patch_once(c, r"(size_t Circuit::measure\(\) \{\n)", lambda m: m.group(1) + MEASURE_HOOK,
                   "Circuit::measure")
    c = patch_once(c, r"(std::vector<size_t> Circuit::sample\(int numShots\)\s*\{\n)",
                   lambda m: m.group(1) + SAMPLE_HOOK, "Circuit::sample")
    with open(os.path.join(out, "Circuit.cpp"), "w") as f:
        f.write(c)


if __name__ == "__main__":
    main()
