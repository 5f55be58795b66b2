// CircuitUnitaryOperationB200.cpp -- see the header.
#include "CircuitUnitaryOperationB200.h"

#include <chrono>
#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>

#include "StateVector.h"

CircuitUnitaryOperationB200::CircuitUnitaryOperationB200(int device)
    : ctx_(nullptr), state_(nullptr), bound_(nullptr), hostDirty_(false)
{
    check(qse_ctx_create(device, &ctx_), "qse_ctx_create");
}

CircuitUnitaryOperationB200::~CircuitUnitaryOperationB200()
{
    if (state_) qse_state_destroy(state_);
    if (ctx_) qse_ctx_destroy(ctx_);
}

void CircuitUnitaryOperationB200::check(int status, const char* what) const
{
    if (status != QSE_OK) throw std::runtime_error(std::string(what) + ": " + qse_last_error());
}

// CircuitUnitaryOperationGPU.cu:158-180: (re)bind, (re)allocate, upload when needed.
void CircuitUnitaryOperationB200::ensureOnDevice(StateVector& sv)
{
    const bool same = (bound_ == &sv) && state_;
    if (same && !hostDirty_) return;
    if (bound_ && bound_ != &sv && state_ && !hostDirty_) flush();
    const uint32_t n = static_cast<uint32_t>(sv.qubits());
    if (state_ && qse_state_qubits(state_) != n) {
        qse_state_destroy(state_);
        state_ = nullptr;
    }
    if (!state_) check(qse_state_create(ctx_, n, &state_), "qse_state_create");
    check(qse_state_upload(state_, reinterpret_cast<const double*>(sv.getRawPtr())), "qse_state_upload");
    bound_ = &sv;
    hostDirty_ = false;
}

void CircuitUnitaryOperationB200::flush()
{
    if (!bound_ || !state_ || hostDirty_) return;
    check(qse_state_download(state_, reinterpret_cast<double*>(bound_->getRawPtr())), "qse_state_download");
}

void CircuitUnitaryOperationB200::markHostDirty() { hostDirty_ = true; }

void CircuitUnitaryOperationB200::timed(const char* label, int status)
{
    check(status, label);
}

#define QSE_TIMED(label, call)                                                                      \
    do {                                                                                            \
        auto t0_ = std::chrono::high_resolution_clock::now();                                       \
        timed(label, (call));                                                                       \
        if (print_steps) {                                                                          \
            check(qse_ctx_synchronize(ctx_), "qse_ctx_synchronize");                                \
            std::chrono::duration<double, std::milli> ms_ = std::chrono::high_resolution_clock::now() - t0_; \
            std::cout << label << " applied in: " << ms_.count() << " ms (GPU)\n";                  \
        }                                                                                           \
    } while (0)

void CircuitUnitaryOperationB200::applyGate(StateVector& sv, const Gate2x2& g, size_t q)
{
    ensureOnDevice(sv);
    double m[8] = {g.data[0][0].real(), g.data[0][0].imag(), g.data[0][1].real(), g.data[0][1].imag(),
                   g.data[1][0].real(), g.data[1][0].imag(), g.data[1][1].real(), g.data[1][1].imag()};
    QSE_TIMED("Gate", qse_apply_gate2x2(state_, m, uint32_t(q)));
}

void CircuitUnitaryOperationB200::applyCNOT(StateVector& sv, size_t control, size_t target)
{
    ensureOnDevice(sv);
    QSE_TIMED("CNOT", qse_apply_cnot(state_, uint32_t(control), uint32_t(target)));
}

void CircuitUnitaryOperationB200::applyPauliX(StateVector& sv, size_t q)
{
    ensureOnDevice(sv);
    QSE_TIMED("PauliX", qse_apply_x(state_, uint32_t(q)));
}

void CircuitUnitaryOperationB200::applyPauliY(StateVector& sv, size_t q)
{
    ensureOnDevice(sv);
    QSE_TIMED("PauliY", qse_apply_y(state_, uint32_t(q)));
}

void CircuitUnitaryOperationB200::applyPauliZ(StateVector& sv, size_t q)
{
    ensureOnDevice(sv);
    QSE_TIMED("PauliZ", qse_apply_z(state_, uint32_t(q)));
}

void CircuitUnitaryOperationB200::applyPhase(StateVector& sv, size_t q, double theta)
{
    ensureOnDevice(sv);
    QSE_TIMED("Phase", qse_apply_phase(state_, uint32_t(q), theta));
}

void CircuitUnitaryOperationB200::applyRotateX(StateVector& sv, size_t q, double theta)
{
    ensureOnDevice(sv);
    QSE_TIMED("RotateX", qse_apply_rx(state_, uint32_t(q), theta));
}

void CircuitUnitaryOperationB200::applyRotateY(StateVector& sv, size_t q, double theta)
{
    ensureOnDevice(sv);
    QSE_TIMED("RotateY", qse_apply_ry(state_, uint32_t(q), theta));
}

void CircuitUnitaryOperationB200::applyRotateZ(StateVector& sv, size_t q, double theta)
{
    ensureOnDevice(sv);
    QSE_TIMED("RotateZ", qse_apply_rz(state_, uint32_t(q), theta));
}

void CircuitUnitaryOperationB200::applyHadamard(StateVector& sv, size_t q)
{
    ensureOnDevice(sv);
    QSE_TIMED("Hadamard", qse_apply_h(state_, uint32_t(q)));
}

void CircuitUnitaryOperationB200::applyCPhase(StateVector& sv, size_t control, size_t target, double theta)
{
    ensureOnDevice(sv);
    QSE_TIMED("CPhase", qse_apply_cphase(state_, uint32_t(control), uint32_t(target), theta));
}

void CircuitUnitaryOperationB200::applyMCPhase(StateVector& sv, const std::vector<size_t>& controls, size_t target,
                                               double theta)
{
    ensureOnDevice(sv);
    std::vector<uint32_t> c(controls.begin(), controls.end());
    QSE_TIMED("MCPhase", qse_apply_mcphase(state_, c.data(), c.size(), uint32_t(target), theta));
}

void CircuitUnitaryOperationB200::applySwap(StateVector& sv, size_t q0, size_t q1)
{
    ensureOnDevice(sv);
    QSE_TIMED("Swap", qse_apply_swap(state_, uint32_t(q0), uint32_t(q1)));
}

bool CircuitUnitaryOperationB200::executeProgram(StateVector& sv, const std::vector<GateCommand>& commands)
{
    ensureOnDevice(sv);
    std::vector<qse_op> ops;
    ops.reserve(commands.size());
    for (const GateCommand& c : commands) {
        qse_op op{};
        op.type = static_cast<int32_t>(c.type);
        op.target = static_cast<uint32_t>(c.target);
        op.control = static_cast<uint32_t>(c.control);
        op.param = -1;
        op.theta = c.theta;
        for (size_t q : c.controls_list) op.controls |= uint64_t(1) << q;
        ops.push_back(op);
    }
    qse_exec_stats stats{};
    QSE_TIMED("Program", qse_execute(state_, ops.data(), ops.size(), nullptr, 0, nullptr, nullptr, 0, &stats));
    return true;
}

bool CircuitUnitaryOperationB200::sample(StateVector& sv, const double* uniforms, size_t shots,
                                         std::vector<size_t>& out)
{
    ensureOnDevice(sv);
    std::vector<uint64_t> idx(shots);
    if (shots) check(qse_sample(state_, uniforms, shots, 0, idx.data()), "qse_sample");
    out.assign(idx.begin(), idx.end());
    return true;
}

bool CircuitUnitaryOperationB200::measure(StateVector& sv, double u, size_t& out)
{
    ensureOnDevice(sv);
    uint64_t idx = 0;
    check(qse_measure(state_, u, &idx), "qse_measure");
    out = static_cast<size_t>(idx);
    return true;
}
