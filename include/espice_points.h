/*
 * espice_points.h: the reference's points API (include/espice.h:286-360:
 * espice_append_points, espice_copy_point_measures, espice_release_points,
 * espice_lane_width; src/c_api.zig:599-667) over the sweep-lane library
 * (libespice_lanes.so).
 *
 * A points problem holds one frozen circuit (the template), its live
 * parameters (the slots each point sets, espice_create_options.live_params),
 * one analysis (an operating point or a transient) and the named results a
 * point reports: the transient's .meas cards, or unknowns at the operating
 * point. Appended points queue; they run together as lanes of one device
 * launch (up to lane_width points a launch) when their results are first
 * copied, so espice_lane_width reports more than 1 here. The reference's
 * deck front end (espice_create from a netlist) is not part of this
 * library: a caller builds the circuit with esl_circuit.
 *
 * Status codes are the reference's espice_status values; per-point reasons
 * its espice_reason values.
 */
#ifndef ESPICE_POINTS_H
#define ESPICE_POINTS_H

#include <stddef.h>
#include <stdint.h>

#include "espice_lanes.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { /* espice_status (include/espice.h:34-37) */
    ESL_PTS_OK = 0,
    ESL_PTS_INVALID_ARGUMENT = 1,
    ESL_PTS_OUT_OF_MEMORY = 3,
    ESL_PTS_INVALID_QUERY = 4,
    ESL_PTS_RESULT_UNAVAILABLE = 5,
    ESL_PTS_FAILED = 6,
    ESL_PTS_ABI_MISMATCH = 7
};

enum { /* espice_reason (include/espice.h:260-283) */
    ESL_REASON_OK = 0,
    ESL_REASON_NO_CONVERGENCE = 1,
    ESL_REASON_TIMESTEP_TOO_SMALL = 2,
    ESL_REASON_SINGULAR_MATRIX = 3,
    ESL_REASON_MEASURE_UNRESOLVED = 5,
    ESL_REASON_OTHER = 255
};

enum { ESL_POINTS_OP = 0, ESL_POINTS_TRAN = 1 };
enum { ESL_RESULT_MEASURE = 0, ESL_RESULT_UNKNOWN = 1 };

/* A named result of every point (names compare case-insensitively): card
 * `index` of the transient's measures, or unknown `index` at the operating
 * point. */
typedef struct {
    const char *name;
    uint32_t kind;
    uint32_t index;
} esl_points_result;

typedef struct {
    const esl_circuit *circuit;
    const esl_slot *live;     /* the live parameters, values[k] of a point sets live[k] */
    uint32_t n_live;
    uint32_t analysis;        /* ESL_POINTS_OP or ESL_POINTS_TRAN */
    esl_newton_opts newton;   /* the operating point's Newton options */
    esl_tran_opts tran;       /* the transient's options */
    const esl_measure *measures; /* the transient's .meas cards (at most 32) */
    uint32_t n_measures;
    const esl_points_result *results;
    uint32_t n_results;
    int device;
    uint32_t lane_width;      /* points a launch runs together (0: 4096) */
} esl_points_config;

/* espice_bytes and espice_points_options with the reference's layout
 * (40 bytes through warm_start on LP64, then tangent_step). */
typedef struct { const char *data; size_t len; } esl_bytes;
typedef struct {
    size_t struct_size;
    esl_bytes abort_measure;
    double abort_after;
    uint8_t measures_only;
    uint8_t early_stop;   /* transient: a lane ends once its measures resolve */
    uint8_t warm_start;   /* operating point: 1 from the template's nominal OP, 0 cold (a
                             transient's lanes solve their operating point cold) */
    double tangent_step;
} esl_points_options;

typedef struct esl_points esl_points;

/* Builds the template (esl_create). INVALID_ARGUMENT for a null pointer, a
 * live slot outside the circuit, more than 32 measures, a result name given
 * twice or a result of the other analysis; FAILED without a device. */
int32_t esl_points_create(const esl_points_config *config, esl_points **out);
int32_t esl_points_destroy(esl_points *p);
const char *esl_points_error(const esl_points *p);

/* espice_append_points: count points, values [count][n_live]; *first_id
 * receives point 0's id (ids are consecutive). options NULL: every flag 0.
 * ESL_PTS_ABI_MISMATCH for a struct_size short of 40; INVALID_ARGUMENT for
 * count 0, a flag above 1, a negative or infinite abort_after, an
 * abort_after other than NaN (the lanes run each transient to its end or to
 * its measures' resolution), or a tangent_step above 0 (tangents are
 * unavailable on a GPU backend, as in the reference). */
int32_t esl_points_append(esl_points *p, const double *values, size_t count, const esl_points_options *options,
                          uint32_t *first_id);

/* espice_copy_point_measures: runs the points not yet run (lane batches of
 * up to lane_width), then copies the results `names` of count points from
 * first_id into out [count][measure_count] and each point's reason into
 * reasons[count]: NO_CONVERGENCE / SINGULAR_MATRIX / TIMESTEP_TOO_SMALL for
 * a failed point (its values NaN), MEASURE_UNRESOLVED when a requested
 * measure has no value. INVALID_ARGUMENT for a name no result has;
 * INVALID_QUERY for ids outside the appended points; RESULT_UNAVAILABLE for
 * released points. Nothing is written on failure. */
int32_t esl_points_copy_measures(esl_points *p, uint32_t first_id, size_t count, const esl_bytes *names,
                                 size_t measure_count, double *out, uint32_t *reasons);

/* espice_release_points: frees the results of count points from first_id. */
int32_t esl_points_release(esl_points *p, uint32_t first_id, size_t count);

/* espice_lane_width: the points a launch runs together. */
int32_t esl_points_lane_width(esl_points *p, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
