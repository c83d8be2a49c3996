/* TEST INFRASTRUCTURE (oracle), not product code. MOS1 (models/mos1.va). */
#include "orc_internal.h"

#include <string.h>

void mos1_derive(const double *prm, double *der) {
    (void)prm;
    memset(der, 0, sizeof(double) * ORC_NDER);
}

void mos1_eval(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *lim, const double *st, const sim_t *sim, devout_t *o) {
    (void)nd; (void)prm; (void)der; (void)x; (void)lim; (void)st; (void)sim;
    memset(o, 0, sizeof(*o));
}

int mos1_limit(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *x_old, const double *lim_old, double *lim_new) {
    (void)nd; (void)prm; (void)der; (void)x; (void)x_old; (void)lim_old; (void)lim_new;
    return 0;
}

int mos1_seed(const uint32_t *nd, const double *prm, const double *der, const double *x, double *lim) {
    (void)nd; (void)prm; (void)der; (void)x; (void)lim;
    return 0;
}
