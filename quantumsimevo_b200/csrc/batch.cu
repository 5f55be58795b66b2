// batch.cu -- batched forward + adjoint of many small circuits (placeholder until the
// persistent kernel lands; every entry point reports QSE_ERR_UNSUPPORTED).
#include "qse_internal.h"

extern "C" {
int qse_batch_create(qse_ctx*, const qse_batch_circuit*, size_t, qse_batch** out)
{
    if (out) *out = nullptr;
    return QSE_ERR_UNSUPPORTED;
}
int qse_batch_destroy(qse_batch*) { return QSE_OK; }
int qse_batch_run(qse_batch*, const double*, double*, double*) { return QSE_ERR_UNSUPPORTED; }
int qse_batch_run_device(qse_batch*, const double*, double*, double*) { return QSE_ERR_UNSUPPORTED; }
int qse_batch_total_params(const qse_batch*, size_t* n)
{
    if (n) *n = 0;
    return QSE_ERR_UNSUPPORTED;
}
int qse_batch_autotune(qse_batch*, const char*) { return QSE_ERR_UNSUPPORTED; }
int qse_batch_use_graph(qse_batch*, int) { return QSE_ERR_UNSUPPORTED; }
}
