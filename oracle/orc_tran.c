/* TEST INFRASTRUCTURE (oracle), not product code. Transient (tran.zig). */
#include "orc_internal.h"
#include "orc_ckt.h"

int orc_tran(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
             const double *values, uint32_t n_lanes, const orc_tran_opts *topts,
             const double *x0, const uint32_t *probe_nodes, uint32_t n_probes,
             uint32_t max_pts, double *out_t, double *out_v, uint32_t *n_pts_out,
             uint32_t *stats, double *x_final) {
    (void)c; (void)slots; (void)n_slots; (void)values; (void)n_lanes; (void)topts; (void)x0;
    (void)probe_nodes; (void)n_probes; (void)max_pts; (void)out_t; (void)out_v; (void)n_pts_out;
    (void)stats; (void)x_final;
    return -1;
}
