// The points API (include/espice_points.h) over the sweep-lane library: the
// reference's espice_append_points / espice_copy_point_measures /
// espice_release_points / espice_lane_width (src/c_api.zig:599-667) with the
// points run as lanes. Appended points queue; the first copy that needs
// them runs every queued point, grouped by their run options, in launches
// of up to lane_width lanes (esl_set_lanes, then esl_dc_solve or
// esl_tran_meas_device), and keeps each point's named results and reason.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/espice_lanes.h"
#include "../../../include/espice_points.h"

namespace {

constexpr uint32_t kDefaultLaneWidth = 4096;
constexpr size_t kOptionsAbiBytes = 40;  // espice_points_options through warm_start, on LP64

std::string lower(const char* s, size_t len) {
  std::string out(s, len);
  for (char& c : out) c = char(std::tolower(static_cast<unsigned char>(c)));
  return out;
}

struct Point {
  std::vector<double> values;
  uint8_t early_stop = 0, warm_start = 0;
  bool done = false, released = false;
  uint32_t reason = ESL_REASON_OK;
  std::vector<double> results;  // one per configured result
};

}  // namespace

struct esl_points {
  esl_ctx* ctx = nullptr;
  int device = 0;
  std::string err;
  uint32_t analysis = ESL_POINTS_OP, lane_width = kDefaultLaneWidth, n = 0;
  std::vector<esl_slot> live;
  esl_newton_opts newton{};
  esl_tran_opts tran{};
  std::vector<esl_measure> meas;
  struct Result {
    std::string name;
    uint32_t kind, index;
  };
  std::vector<Result> results;
  std::vector<double> x_nominal;
  bool have_nominal = false;
  std::vector<Point> pts;

  int32_t fail(int32_t code, const std::string& what) {
    err = what;
    return code;
  }
};

namespace {

// The template's nominal operating point (a warm start's x0).
int32_t ensure_nominal(esl_points* p) {
  if (p->have_nominal) return ESL_PTS_OK;
  if (esl_set_lanes(p->ctx, nullptr, 0, nullptr, 1) != ESL_OK)
    return p->fail(ESL_PTS_FAILED, std::string("nominal point: ") + esl_last_error(p->ctx));
  std::vector<double> x(p->n);
  uint32_t it = 0, st = 0;
  if (esl_dc_solve(p->ctx, &p->newton, nullptr, x.data(), &it, &st, nullptr) != ESL_OK)
    return p->fail(ESL_PTS_FAILED, std::string("nominal point: ") + esl_last_error(p->ctx));
  if (st != ESL_LANE_CONVERGED) return p->fail(ESL_PTS_FAILED, "the template's nominal operating point did not converge");
  p->x_nominal = x;
  p->have_nominal = true;
  return ESL_PTS_OK;
}

uint32_t tran_reason(uint32_t status) {
  switch (status) {
    case ESL_TRAN_DONE:
    case ESL_TRAN_RESOLVED:
      return ESL_REASON_OK;
    case ESL_TRAN_UNDERFLOW:
      return ESL_REASON_TIMESTEP_TOO_SMALL;
    case ESL_TRAN_OP_FAILED:
      return ESL_REASON_NO_CONVERGENCE;
    default:
      return ESL_REASON_OTHER;
  }
}

// One launch over the points `ids` (same run options, at most lane_width).
int32_t run_batch(esl_points* p, const std::vector<uint32_t>& ids) {
  const uint32_t N = uint32_t(ids.size()), nl = uint32_t(p->live.size());
  std::vector<double> values(size_t(N) * std::max<uint32_t>(nl, 1));
  for (uint32_t l = 0; l < N; ++l)
    std::copy(p->pts[ids[l]].values.begin(), p->pts[ids[l]].values.end(), values.begin() + size_t(l) * nl);
  const Point& first = p->pts[ids[0]];
  if (first.warm_start && p->analysis == ESL_POINTS_OP)
    if (int32_t rc = ensure_nominal(p)) return rc;
  if (esl_set_lanes(p->ctx, p->live.data(), nl, nl ? values.data() : nullptr, N) != ESL_OK)
    return p->fail(ESL_PTS_FAILED, esl_last_error(p->ctx));
  const size_t R = p->results.size();
  if (p->analysis == ESL_POINTS_OP) {
    std::vector<double> x0, x(size_t(N) * p->n);
    if (first.warm_start) {
      x0.resize(size_t(N) * p->n);
      for (uint32_t l = 0; l < N; ++l) std::copy(p->x_nominal.begin(), p->x_nominal.end(), x0.begin() + size_t(l) * p->n);
    }
    std::vector<uint32_t> it(N), st(N);
    if (esl_dc_solve(p->ctx, &p->newton, x0.empty() ? nullptr : x0.data(), x.data(), it.data(), st.data(), nullptr) !=
        ESL_OK)
      return p->fail(ESL_PTS_FAILED, esl_last_error(p->ctx));
    for (uint32_t l = 0; l < N; ++l) {
      Point& pt = p->pts[ids[l]];
      pt.reason = st[l] == ESL_LANE_CONVERGED ? ESL_REASON_OK
                  : st[l] == ESL_LANE_SINGULAR ? ESL_REASON_SINGULAR_MATRIX
                                               : ESL_REASON_NO_CONVERGENCE;
      pt.results.assign(R, std::numeric_limits<double>::quiet_NaN());
      if (pt.reason == ESL_REASON_OK)
        for (size_t r = 0; r < R; ++r) pt.results[r] = x[size_t(l) * p->n + p->results[r].index];
      pt.done = true;
    }
    return ESL_PTS_OK;
  }
  // transient with streamed measures: device buffers for the launch
  const uint32_t M = uint32_t(p->meas.size());
  double *d_x = nullptr, *d_v = nullptr;
  uint32_t* d_s = nullptr;
  auto release = [&]() {
    cudaFree(d_x);
    cudaFree(d_v);
    cudaFree(d_s);
  };
  if (cudaMalloc(&d_x, size_t(N) * p->n * 8) != cudaSuccess ||
      cudaMalloc(&d_v, size_t(N) * std::max<uint32_t>(M, 1) * 8) != cudaSuccess ||
      cudaMalloc(&d_s, size_t(N) * ESL_TS_N * 4) != cudaSuccess) {
    release();
    return p->fail(ESL_PTS_OUT_OF_MEMORY, "device buffers for a batch of points");
  }
  const int32_t rc = esl_tran_meas_device(p->ctx, &p->tran, p->meas.data(), M, first.early_stop, d_x, d_s, d_v, nullptr);
  std::vector<double> vals(size_t(N) * std::max<uint32_t>(M, 1));
  std::vector<uint32_t> stats(size_t(N) * ESL_TS_N);
  if (rc == ESL_OK) {
    cudaMemcpy(vals.data(), d_v, vals.size() * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(stats.data(), d_s, stats.size() * 4, cudaMemcpyDeviceToHost);
  }
  release();
  if (rc != ESL_OK) return p->fail(ESL_PTS_FAILED, esl_last_error(p->ctx));
  for (uint32_t l = 0; l < N; ++l) {
    Point& pt = p->pts[ids[l]];
    pt.reason = tran_reason(stats[size_t(l) * ESL_TS_N + ESL_TS_STATUS]);
    pt.results.assign(R, std::numeric_limits<double>::quiet_NaN());
    if (pt.reason == ESL_REASON_OK)
      for (size_t r = 0; r < R; ++r) pt.results[r] = vals[size_t(l) * M + p->results[r].index];
    pt.done = true;
  }
  return ESL_PTS_OK;
}

// Every queued point, grouped by run options, in launches of lane_width.
int32_t run_pending(esl_points* p) {
  std::map<std::pair<uint8_t, uint8_t>, std::vector<uint32_t>> groups;
  for (uint32_t id = 0; id < p->pts.size(); ++id)
    if (!p->pts[id].done && !p->pts[id].released) groups[{p->pts[id].early_stop, p->pts[id].warm_start}].push_back(id);
  for (auto& g : groups)
    for (size_t at = 0; at < g.second.size(); at += p->lane_width) {
      const std::vector<uint32_t> ids(g.second.begin() + at,
                                      g.second.begin() + std::min(g.second.size(), at + p->lane_width));
      if (int32_t rc = run_batch(p, ids)) return rc;
    }
  return ESL_PTS_OK;
}

}  // namespace

extern "C" {

int32_t esl_points_create(const esl_points_config* c, esl_points** out) {
  if (!c || !out || !c->circuit || (c->n_live && !c->live) || (c->n_results && !c->results) ||
      c->analysis > ESL_POINTS_TRAN || (c->n_measures && !c->measures) || c->n_measures > 32)
    return ESL_PTS_INVALID_ARGUMENT;
  *out = nullptr;
  auto p = std::make_unique<esl_points>();
  p->device = c->device;
  p->analysis = c->analysis;
  p->lane_width = c->lane_width ? c->lane_width : kDefaultLaneWidth;
  p->live.assign(c->live, c->live + c->n_live);
  p->newton = c->newton;
  p->tran = c->tran;
  p->meas.assign(c->measures, c->measures + c->n_measures);
  for (uint32_t r = 0; r < c->n_results; ++r) {
    const esl_points_result& res = c->results[r];
    if (!res.name) return ESL_PTS_INVALID_ARGUMENT;
    if (res.kind == ESL_RESULT_MEASURE ? (c->analysis != ESL_POINTS_TRAN || res.index >= c->n_measures)
                                       : (c->analysis != ESL_POINTS_OP || res.index >= c->circuit->n))
      return ESL_PTS_INVALID_ARGUMENT;
    const std::string key = lower(res.name, std::strlen(res.name));
    for (const auto& e : p->results)
      if (e.name == key) return ESL_PTS_INVALID_ARGUMENT;
    p->results.push_back({key, res.kind, res.index});
  }
  esl_options o{c->device, 0};
  const int32_t rc = esl_create(c->circuit, &o, &p->ctx);
  if (rc != ESL_OK) {
    esl_destroy(p->ctx);
    return rc == ESL_NO_DEVICE || rc == ESL_DEVICE_FAULT ? ESL_PTS_FAILED : ESL_PTS_INVALID_ARGUMENT;
  }
  p->n = c->circuit->n;
  // the live slots against the template (placeholder values; each run sets its own)
  std::vector<double> probe(std::max<uint32_t>(c->n_live, 1), 1.0);
  if (esl_set_lanes(p->ctx, c->live, c->n_live, c->n_live ? probe.data() : nullptr, 1) != ESL_OK) {
    esl_destroy(p->ctx);
    return ESL_PTS_INVALID_ARGUMENT;
  }
  *out = p.release();
  return ESL_PTS_OK;
}

int32_t esl_points_destroy(esl_points* p) {
  if (!p) return ESL_PTS_OK;
  esl_destroy(p->ctx);
  delete p;
  return ESL_PTS_OK;
}

const char* esl_points_error(const esl_points* p) { return p ? p->err.c_str() : "no points problem"; }

int32_t esl_points_append(esl_points* p, const double* values, size_t count, const esl_points_options* o,
                          uint32_t* first_id) {
  if (!p) return ESL_PTS_INVALID_ARGUMENT;
  if (!first_id || count == 0 || (!p->live.empty() && !values)) return p->fail(ESL_PTS_INVALID_ARGUMENT, "null argument or no points");
  uint8_t early = 0, warm = 0;
  if (o) {
    if (o->struct_size < kOptionsAbiBytes) return p->fail(ESL_PTS_ABI_MISMATCH, "espice_points_options is 40 bytes or more");
    if (o->measures_only > 1 || o->early_stop > 1 || o->warm_start > 1 || o->abort_after < 0 ||
        std::isinf(o->abort_after))
      return p->fail(ESL_PTS_INVALID_ARGUMENT, "an options flag above 1, or a negative or infinite abort_after");
    if (!std::isnan(o->abort_after))
      return p->fail(ESL_PTS_INVALID_ARGUMENT, "abort_after: the lanes run each transient to its end or its measures");
    if (o->struct_size >= sizeof(esl_points_options) && !(o->tangent_step == 0.0))
      return p->fail(ESL_PTS_INVALID_ARGUMENT, "TangentsUnavailable: no tangents on a GPU backend");
    early = o->early_stop;
    warm = o->warm_start;
  }
  const size_t nl = p->live.size();
  for (size_t k = 0; k < count * nl; ++k)
    if (!std::isfinite(values[k])) return p->fail(ESL_PTS_INVALID_ARGUMENT, "a non-finite parameter value");
  *first_id = uint32_t(p->pts.size());
  for (size_t k = 0; k < count; ++k) {
    Point pt;
    pt.values.assign(values + k * nl, values + (k + 1) * nl);
    pt.early_stop = early;
    pt.warm_start = warm;
    p->pts.push_back(std::move(pt));
  }
  return ESL_PTS_OK;
}

int32_t esl_points_copy_measures(esl_points* p, uint32_t first_id, size_t count, const esl_bytes* names,
                                 size_t measure_count, double* out, uint32_t* reasons) {
  if (!p) return ESL_PTS_INVALID_ARGUMENT;
  if ((measure_count && (!names || !out)) || (count && !reasons)) return p->fail(ESL_PTS_INVALID_ARGUMENT, "null argument");
  std::vector<size_t> which(measure_count);
  for (size_t m = 0; m < measure_count; ++m) {
    if (!names[m].data && names[m].len) return p->fail(ESL_PTS_INVALID_ARGUMENT, "null measure name");
    const std::string key = lower(names[m].data ? names[m].data : "", names[m].len);
    size_t r = 0;
    while (r < p->results.size() && p->results[r].name != key) ++r;
    if (r == p->results.size()) return p->fail(ESL_PTS_INVALID_ARGUMENT, "UnknownMeasure: " + key);
    which[m] = r;
  }
  if (size_t(first_id) + count > p->pts.size()) return p->fail(ESL_PTS_INVALID_QUERY, "points beyond those appended");
  for (size_t k = 0; k < count; ++k)
    if (p->pts[first_id + k].released) return p->fail(ESL_PTS_RESULT_UNAVAILABLE, "a released point");
  if (int32_t rc = run_pending(p)) return rc;
  for (size_t k = 0; k < count; ++k) {
    const Point& pt = p->pts[first_id + k];
    uint32_t reason = pt.reason;
    for (size_t m = 0; m < measure_count; ++m) {
      const double v = pt.results[which[m]];
      out[k * measure_count + m] = v;
      if (reason == ESL_REASON_OK && std::isnan(v) && p->results[which[m]].kind == ESL_RESULT_MEASURE)
        reason = ESL_REASON_MEASURE_UNRESOLVED;
    }
    reasons[k] = reason;
  }
  return ESL_PTS_OK;
}

int32_t esl_points_release(esl_points* p, uint32_t first_id, size_t count) {
  if (!p) return ESL_PTS_INVALID_ARGUMENT;
  if (size_t(first_id) + count > p->pts.size()) return p->fail(ESL_PTS_INVALID_QUERY, "points beyond those appended");
  for (size_t k = 0; k < count; ++k) {
    Point& pt = p->pts[first_id + k];
    pt.released = true;
    std::vector<double>().swap(pt.results);
  }
  return ESL_PTS_OK;
}

int32_t esl_points_lane_width(esl_points* p, uint32_t* out) {
  if (!p || !out) return ESL_PTS_INVALID_ARGUMENT;
  *out = p->lane_width;
  return ESL_PTS_OK;
}

}  // extern "C"
