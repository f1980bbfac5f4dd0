// Variational calls on one state: the VQE objective (src/optimization/vqe.rs:63-67),
// ParameterShift::compute_gradient (src/optimization/gradient.rs:44-78) and
// FiniteDifference::compute_gradient (src/optimization/gradient.rs:96-125).
//
// This is the plain per-circuit path: every energy is one Circuit::execute from
// |0...0> (fused passes) followed by one Pauli-sum reduction, exactly as the
// reference re-simulates each shifted circuit.  The batched engine (batch.cu)
// runs the same 2P+1 circuits of many instances in one persistent launch.
#include "lq_internal.h"

namespace lq {

static int check_variational(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                             int nparams, const lq_pauli_term *terms, int nterms, int yconv) {
    LQ_TRY(check_state(work));
    if (nops < 0 || (nops > 0 && !ops)) return set_error(LQ_ERR_INVALID_ARG, "bad op list");
    if (nparams < 0 || (nparams > 0 && !theta))
        return set_error(LQ_ERR_INVALID_ARG, "bad parameter vector");
    if (nterms < 0 || (nterms > 0 && !terms)) return set_error(LQ_ERR_INVALID_ARG, "bad terms");
    if (yconv != LQ_Y_REFERENCE && yconv != LQ_Y_TEXTBOOK)
        return set_error(LQ_ERR_INVALID_ARG, "unknown Y convention %d", yconv);
    for (int i = 0; i < nops; ++i) LQ_TRY(validate_gate(&ops[i], work->n, nparams));
    return LQ_OK;
}

static int energy_at(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                     int nparams, const lq_pauli_term *terms, int nterms, int yconv, double *e) {
    LQ_TRY(lq_state_set_basis(work, 0));
    LQ_TRY(apply_circuit_impl(work, ops, nops, theta, nparams, LQ_EXEC_FUSED));
    if (nterms == 0) {
        *e = 0.0;
        return LQ_OK;
    }
    return expectation_impl(work, terms, nterms, yconv, e, nullptr);
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_ansatz_energy(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                     int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                     double *energy) {
    LQ_TRY(check_variational(work, ops, nops, theta, nparams, terms, nterms, y_convention));
    if (!energy) return set_error(LQ_ERR_INVALID_ARG, "null output");
    return energy_at(work, ops, nops, theta, nparams, terms, nterms, y_convention, energy);
}

int lq_parameter_shift(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                       int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                       double shift, double *grad) {
    LQ_TRY(check_variational(work, ops, nops, theta, nparams, terms, nterms, y_convention));
    if (nparams > 0 && !grad) return set_error(LQ_ERR_INVALID_ARG, "null gradient output");
    std::vector<double> p(theta, theta + nparams);
    for (int i = 0; i < nparams; ++i) {
        double ep, em;
        p[i] = theta[i] + shift;
        LQ_TRY(energy_at(work, ops, nops, p.data(), nparams, terms, nterms, y_convention, &ep));
        p[i] = theta[i] - shift;
        LQ_TRY(energy_at(work, ops, nops, p.data(), nparams, terms, nterms, y_convention, &em));
        p[i] = theta[i];
        grad[i] = (ep - em) / 2.0;
    }
    return LQ_OK;
}

int lq_finite_difference(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                         int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                         double epsilon, double *grad) {
    LQ_TRY(check_variational(work, ops, nops, theta, nparams, terms, nterms, y_convention));
    if (nparams > 0 && !grad) return set_error(LQ_ERR_INVALID_ARG, "null gradient output");
    std::vector<double> p(theta, theta + nparams);
    double fx;
    LQ_TRY(energy_at(work, ops, nops, theta, nparams, terms, nterms, y_convention, &fx));
    for (int i = 0; i < nparams; ++i) {
        double fp;
        p[i] = theta[i] + epsilon;
        LQ_TRY(energy_at(work, ops, nops, p.data(), nparams, terms, nterms, y_convention, &fp));
        p[i] = theta[i];
        grad[i] = (fp - fx) / epsilon;
    }
    return LQ_OK;
}

}  // extern "C"
