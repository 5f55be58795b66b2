// CircuitUnitaryOperationB200.h -- drop-in backend for QuantumSimEvo's
// ICircuitUnitaryOperation (QuantumSimEvo/ICircuitUnitaryOperation.h:6-35),
// standing in for CircuitUnitaryOperationGPU (CircuitUnitaryOperationGPU.h:10-48).
//
// Compiled inside the reference tree: it includes the reference's own
// interface header and forwards every call to the C ABI of libqse_b200.so
// (include/qse_b200.h).  Mirror protocol as the reference GPU backend
// (CircuitUnitaryOperationGPU.cu:158-192): the device copy is authoritative
// after any apply*, flush() copies it into the bound StateVector, and
// markHostDirty() forces a re-upload before the next gate.  Errors throw
// std::runtime_error instead of aborting the process.
#ifndef CIRCUIT_UNITARY_OPERATION_B200_H
#define CIRCUIT_UNITARY_OPERATION_B200_H

#include <cstddef>
#include <vector>

#include "ICircuitUnitaryOperation.h"
#include "Structurs.h"
#include "qse_b200.h"

class CircuitUnitaryOperationB200 : public ICircuitUnitaryOperation {
public:
    explicit CircuitUnitaryOperationB200(int device = 0);
    ~CircuitUnitaryOperationB200() override;

    void applyGate(StateVector& sv, const Gate2x2& gate, size_t q) override;
    void applyCNOT(StateVector& sv, size_t control, size_t target) override;
    void applyPauliX(StateVector& sv, size_t q) override;
    void applyPauliY(StateVector& sv, size_t q) override;
    void applyPauliZ(StateVector& sv, size_t q) override;
    void applyPhase(StateVector& sv, size_t q, double theta) override;
    void applyRotateX(StateVector& sv, size_t q, double theta) override;
    void applyRotateY(StateVector& sv, size_t q, double theta) override;
    void applyRotateZ(StateVector& sv, size_t q, double theta) override;
    void applyHadamard(StateVector& sv, size_t targetQubit) override;
    void applyCPhase(StateVector& sv, size_t control, size_t target, double theta) override;
    void applyMCPhase(StateVector& sv, const std::vector<size_t>& controls, size_t target, double theta) override;
    void applySwap(StateVector& sv, size_t q0, size_t q1) override;

    void flush() override;
    void markHostDirty() override;

    // Optional hooks a Circuit can call when the interface declares them as
    // virtuals with declining defaults (the test build compiles such a patched
    // ICircuitUnitaryOperation.h and Circuit.cpp, oracle/patch_reference.py).
    // Against the unpatched interface they are plain members.  Each returns
    // true: it handled the call.
    //
    // executeProgram: Circuit::execute's whole queue (Circuit.cpp:64-120,
    // noise off) through the fusion planner -- one call, any number of passes.
    bool executeProgram(StateVector& sv, const std::vector<GateCommand>& commands);

    // Circuit::sample / Circuit::measure (StateVector.cpp:77-156) on the device
    // copy, so neither needs the full-state copy to the host.  Each shot / the
    // measurement takes its uniform draw u in [0, 1) from the caller (the
    // reference draws from std::random_device); the outcome is the one
    // StateVector::sample / measure gives for the same draw.  measure()
    // collapses the device copy, which stays authoritative (flush() brings it
    // to the host).
    bool sample(StateVector& sv, const double* uniforms, size_t shots, std::vector<size_t>& out);
    bool measure(StateVector& sv, double u, size_t& out);

    // the C-ABI context (device + stream) this backend runs on
    qse_ctx* context() const { return ctx_; }

private:
    void ensureOnDevice(StateVector& sv);
    void check(int status, const char* what) const;
    void timed(const char* label, int status);

    qse_ctx* ctx_;
    qse_state* state_;
    StateVector* bound_;
    bool hostDirty_;
};

#endif
