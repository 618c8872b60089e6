// extern "C" boundary (include/geneva.h).  Handles own their memory; every
// entry point returns a status and records a message for gva_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/geneva.h"
#include "gva_engine.cuh"
#include "gva_dplan.h"
#include "gva_internal.h"
#include "gva_pool.h"

namespace gva {
const char* last_error_cstr();
}

using namespace gva;

struct gva_db {
    DevDB* dev = nullptr;
    std::string warnings;
};
namespace {
// Runs fn(i) for i in [0, n) on the host's cores (inline below 256 items);
// returns the first failing status, with that worker's message re-raised on
// the calling thread.
template <typename F>
int parallel_for(int n, F fn) {
    const unsigned nth = n < 256 ? 1u : gva::pool_width();
    if (nth == 1) {
        for (int i = 0; i < n; ++i) {
            int st = fn(i);
            if (st) return st;
        }
        return GVA_OK;
    }
    std::vector<int> rc(nth, GVA_OK);
    std::vector<std::string> msg(nth);
    gva::pool_run(nth, [&](unsigned t) {
        for (int i = (int)t; i < n; i += (int)nth) {
            int st = fn(i);
            if (st) {
                rc[t] = st;
                msg[t] = gva::last_error_cstr();
                return;
            }
        }
    });
    for (unsigned t = 0; t < nth; ++t)
        if (rc[t]) return gva::fail(rc[t], msg[t]);
    return GVA_OK;
}
}  // namespace

struct gva_plan {
    Plan plan;
    // steps are lowered per database (labels differ); cache the last lowering
    const gva_db* lowered_for = nullptr;
    std::vector<Step> steps;
};
struct gva_result {
    MatchResult r;
};
struct gva_session {
    BatchSession* ses = nullptr;
    gva_db* db = nullptr;
    std::vector<int> ready;  // completed plans not yet polled
};
struct gva_mine_result {
    std::vector<MinedPattern> pats;
    MineStats stats;
};

namespace {

int steps_for(const gva_plan* p, const gva_db* db, std::vector<Step>& out) {
    return lower_plan(p->plan, db->dev->meta, out);
}

int read_file(const char* path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return fail(GVA_ERR_IO, std::string("cannot open ") + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return GVA_OK;
}

}  // namespace

extern "C" {

const char* gva_last_error(void) { return last_error_cstr(); }

const char* gva_status_string(int s) {
    switch (s) {
        case GVA_OK: return "ok";
        case GVA_ERR_IO: return "i/o error";
        case GVA_ERR_FORMAT: return "format error";
        case GVA_ERR_CUDA: return "cuda error";
        case GVA_ERR_NOMEM: return "out of memory";
        case GVA_ERR_ARG: return "bad argument";
        case GVA_ERR_UNSUPPORTED: return "unsupported";
        case GVA_ERR_CANCELLED: return "cancelled";
        default: return "unknown status";
    }
}

const char* gva_version(void) { return "geneva_b200 0.1 (sm_100a)"; }

uint64_t gva_kernel_launches(void) { return kernel_launches(); }

int gva_result_kernel_stats(const gva_result* res, gva_kernel_stat* out, int cap) {
    if (!res) return -1;
    for (int i = 0; i < K_NUM && i < cap; ++i) {
        memset(&out[i], 0, sizeof out[i]);
        strncpy(out[i].name, kKernelNames[i], sizeof out[i].name - 1);
        out[i].launches = res->r.kstat[i].launches;
        out[i].ms = res->r.kstat[i].ms;
        out[i].bytes = res->r.kstat[i].bytes;
        out[i].rows = res->r.kstat[i].rows;
    }
    return K_NUM;
}

int gva_db_load(const char* mygraph_path, const char* metadata_path, int device, gva_db** out) {
    if (!out || !mygraph_path || !metadata_path) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    HostGraph g;
    std::string warn;
    int st = load_mygraph(mygraph_path, metadata_path, g, &warn);
    if (st) return st;
    DevDB* dev = nullptr;
    st = upload_graph(g, device, dev);
    if (st) return st;
    gva_db* h = new gva_db();
    h->dev = dev;
    h->warnings = warn;
    *out = h;
    return GVA_OK;
}

int gva_db_from_edges(const uint32_t* vertex_labels, uint32_t max_vertex_id, const uint32_t* src, const uint32_t* dst,
                      const uint32_t* edge_labels, uint64_t num_edges, int device, gva_db** out) {
    if (!out) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    HostGraph g;
    int st = graph_from_edges(vertex_labels, max_vertex_id, src, dst, edge_labels, num_edges, g);
    if (st) return st;
    DevDB* dev = nullptr;
    st = upload_graph(g, device, dev);
    if (st) return st;
    gva_db* h = new gva_db();
    h->dev = dev;
    *out = h;
    return GVA_OK;
}

int gva_db_get_info(const gva_db* db, gva_db_info* out) {
    if (!db || !out) return fail(GVA_ERR_ARG, "null argument");
    memset(out, 0, sizeof *out);
    out->max_vertex_id = db->dev->max_id;
    out->num_vertex_labels = db->dev->L;
    out->num_partitions = (uint32_t)db->dev->parts.size();
    out->num_adjacency = db->dev->n_adj;
    out->device_bytes = db->dev->arena_bytes;
    return GVA_OK;
}

int gva_graph_probe(const char* mygraph_path, const char* metadata_path, gva_db_info* out, char* warn, size_t cap) {
    if (!mygraph_path || !metadata_path || !out) return fail(GVA_ERR_ARG, "null argument");
    HostGraph g;
    std::string w;
    int st = load_mygraph(mygraph_path, metadata_path, g, &w);
    if (st) return st;
    memset(out, 0, sizeof *out);
    out->max_vertex_id = g.max_id;
    out->num_vertex_labels = g.num_labels();
    out->num_partitions = (uint32_t)g.parts.size();
    uint64_t bytes = 0;
    for (auto& p : g.parts) {
        out->num_adjacency += p.adj.size();
        bytes += ((p.off.size() * 4 + 255) / 256 + (p.adj.size() * 4 + 4 + 255) / 256) * 256;
    }
    out->device_bytes = bytes + ((uint64_t)g.max_id * 4 + 4 + 255) / 256 * 256;
    if (warn && cap) {
        size_t n = std::min(cap - 1, w.size());
        memcpy(warn, w.data(), n);
        warn[n] = 0;
    }
    return GVA_OK;
}

const char* gva_db_warnings(const gva_db* db) { return db ? db->warnings.c_str() : ""; }

void gva_db_free(gva_db* db) {
    if (!db) return;
    free_devdb(db->dev);
    delete db;
}

int gva_convert_g(const char* g_path, const char* mygraph_path, const char* metadata_path, const char* reorder_path) {
    if (!g_path || !mygraph_path || !metadata_path || !reorder_path) return fail(GVA_ERR_ARG, "null argument");
    return convert_g(g_path, mygraph_path, metadata_path, reorder_path);
}

int gva_plan_batch(const char* const* query_texts, int n, int mode, gva_plan** out, int* status) {
    if (n < 0 || (n > 0 && (!query_texts || !out))) return fail(GVA_ERR_ARG, "null argument");
    for (int i = 0; i < n; ++i) out[i] = nullptr;
    std::vector<int> st(n, GVA_OK);
    std::vector<std::string> msg(n);
    parallel_for(n, [&](int i) {
        if (!query_texts[i]) {
            st[i] = GVA_ERR_ARG;
            msg[i] = "null query text";
            return GVA_OK;
        }
        gva_plan* p = new gva_plan();
        st[i] = plan_from_text(query_texts[i], mode, p->plan);
        if (st[i]) {
            msg[i] = last_error_cstr();
            delete p;
        } else {
            out[i] = p;
        }
        return GVA_OK;  // per-query failures are reported in status, not as the call's
    });
    int first = -1;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (st[i] && first < 0) first = i;
    }
    if (first >= 0) return fail(st[first], "query " + std::to_string(first) + ": " + msg[first]);
    return GVA_OK;
}

int gva_plan_batch_device(int device, const char* const* query_texts, int n, gva_plan** out, int* status) {
    if (n < 0 || (n > 0 && (!query_texts || !out))) return fail(GVA_ERR_ARG, "null argument");
    for (int i = 0; i < n; ++i) out[i] = nullptr;
    std::vector<int> st(n, GVA_OK);
    std::vector<std::string> msg(n);
    std::vector<std::vector<uint32_t>> lab(n), sdl(n);
    parallel_for(n, [&](int i) {
        st[i] = query_texts[i] ? read_query_text(query_texts[i], lab[i], sdl[i]) : fail(GVA_ERR_ARG, "null query text");
        if (st[i]) msg[i] = last_error_cstr();
        return GVA_OK;
    });
    std::vector<DevPlanQuery> dq;
    std::vector<int> slot(n, -1);
    for (int i = 0; i < n; ++i) {
        if (st[i]) continue;
        bool ok = !sdl[i].empty() && lab[i].size() <= (size_t)kDevPlanV && sdl[i].size() / 3 <= (size_t)kDevPlanLines;
        for (size_t e = 0; e + 2 < sdl[i].size() && ok; e += 3)
            ok = sdl[i][e] < lab[i].size() && sdl[i][e + 1] < lab[i].size() && sdl[i][e] != sdl[i][e + 1];
        if (!ok) continue;
        DevPlanQuery q{};
        q.n = (uint32_t)lab[i].size();
        q.lines = (uint32_t)(sdl[i].size() / 3);
        for (uint32_t v = 0; v < q.n; ++v) q.label[v] = lab[i][v];
        for (uint32_t e = 0; e < q.lines; ++e) {
            q.s[e] = (uint8_t)sdl[i][3 * e];
            q.d[e] = (uint8_t)sdl[i][3 * e + 1];
            q.l[e] = sdl[i][3 * e + 2];
        }
        slot[i] = (int)dq.size();
        dq.push_back(q);
    }
    std::vector<DevPlanOut> res(dq.size());
    int rc = plan_on_device(device, nullptr, dq.data(), (uint32_t)dq.size(), res.data());
    if (rc) return rc;
    parallel_for(n, [&](int i) {
        if (st[i]) return GVA_OK;
        gva_plan* p = new gva_plan();
        int r;
        if (slot[i] >= 0 && res[slot[i]].status == DPLAN_OK) {
            thread_local std::unique_ptr<DPlan> dp(new DPlan());
            dplan_from_device(res[slot[i]], *dp);
            r = plan_from_dplan(*dp, lab[i].data(), p->plan);
        } else {
            r = plan_from_query((uint32_t)lab[i].size(), lab[i].data(), sdl[i].data(), sdl[i].size() / 3, GVA_MODE_DV,
                                p->plan);
        }
        if (r) {
            st[i] = r;
            msg[i] = last_error_cstr();
            delete p;
        } else {
            out[i] = p;
        }
        return GVA_OK;
    });
    int first = -1;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (st[i] && first < 0) first = i;
    }
    if (first >= 0) return fail(st[first], "query " + std::to_string(first) + ": " + msg[first]);
    return GVA_OK;
}

int gva_plan_from_text(const char* query_text, int mode, gva_plan** out) {
    if (!out || !query_text) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    gva_plan* p = new gva_plan();
    int st = plan_from_text(query_text, mode, p->plan);
    if (st) {
        delete p;
        return st;
    }
    *out = p;
    return GVA_OK;
}

int gva_plan_from_file(const char* query_path, int mode, gva_plan** out) {
    if (!out || !query_path) return fail(GVA_ERR_ARG, "null argument");
    std::string text;
    int st = read_file(query_path, text);
    if (st) return st;
    return gva_plan_from_text(text.c_str(), mode, out);
}

size_t gva_plan_describe(const gva_plan* plan, char* buf, size_t cap) {
    if (!plan) return 0;
    std::string s = plan->plan.describe();
    if (buf && cap) {
        size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}

int gva_plan_num_phases(const gva_plan* plan) { return plan ? (int)plan->plan.phases.size() : -1; }
int gva_plan_num_vertices(const gva_plan* plan) { return plan ? (int)plan->plan.vnum : -1; }

int gva_plan_column_vertices(const gva_plan* plan, uint32_t* out, int cap) {
    if (!plan) return -1;
    const auto& c = plan->plan.columns;
    for (int i = 0; i < (int)c.size() && i < cap; ++i) out[i] = c[i];
    return (int)c.size();
}

void gva_plan_free(gva_plan* plan) { delete plan; }

int gva_match(gva_db* db, const gva_plan* plan, const gva_match_opts* opts, gva_result** out) {
    if (!db || !plan || !out) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    std::vector<Step> steps;
    int st = steps_for(plan, db, steps);
    if (st) return st;
    gva_match_opts o{};
    if (opts) o = *opts;
    gva_result* r = new gva_result();
    st = run_match(*db->dev, plan->plan, steps, (cudaStream_t)o.stream, o.budget_bytes, o.count_only != 0,
                   o.profile != 0, r->r);
    if (st) {
        delete r;
        return st;
    }
    *out = r;
    return GVA_OK;
}

uint64_t gva_result_num_rows(const gva_result* res) { return res ? res->r.rows : 0; }
int gva_result_num_columns(const gva_result* res) { return res ? (int)res->r.width : -1; }

int gva_result_phase_rows(const gva_result* res, uint64_t* out, int cap) {
    if (!res) return -1;
    const auto& v = res->r.phase_rows;
    for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
    return (int)v.size();
}

const uint32_t* gva_result_device_rows(const gva_result* res) { return res ? res->r.rows_dev : nullptr; }

int gva_result_copy_rows(const gva_result* res, uint32_t* host_dst, uint64_t first_row, uint64_t num_rows) {
    if (!res || (!host_dst && num_rows)) return fail(GVA_ERR_ARG, "null argument");
    if (first_row + num_rows > res->r.rows) return fail(GVA_ERR_ARG, "row range out of bounds");
    if (num_rows == 0) return GVA_OK;
    if (!res->r.rows_dev) return fail(GVA_ERR_ARG, "result holds counts only");
    cudaSetDevice(res->r.device);
    const size_t w = res->r.width;
    cudaError_t e = cudaMemcpyAsync(host_dst, res->r.rows_dev + first_row * w, num_rows * w * 4,
                                    cudaMemcpyDeviceToHost, res->r.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(res->r.stream);
    if (e != cudaSuccess) return fail(GVA_ERR_CUDA, cudaGetErrorString(e));
    return GVA_OK;
}

int gva_result_write_text(const gva_result* res, const char* path) {
    if (!res || !path) return fail(GVA_ERR_ARG, "null argument");
    FILE* f = fopen(path, "w");
    if (!f) return fail(GVA_ERR_IO, std::string("cannot write ") + path);
    const uint64_t chunk = 1 << 22;
    const uint32_t w = res->r.width;
    const unsigned threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<uint32_t> buf;
    std::vector<std::string> parts;
    for (uint64_t r0 = 0; r0 < res->r.rows; r0 += chunk) {
        const uint64_t n = std::min<uint64_t>(chunk, res->r.rows - r0);
        buf.resize(n * w);
        int st = gva_result_copy_rows(res, buf.data(), r0, n);
        if (st) {
            fclose(f);
            return st;
        }
        format_rows(buf.data(), n, w, threads, parts);
        for (const std::string& part : parts)
            if (fwrite(part.data(), 1, part.size(), f) != part.size()) {
                fclose(f);
                return fail(GVA_ERR_IO, std::string("cannot write ") + path);
            }
    }
    if (fclose(f) != 0) return fail(GVA_ERR_IO, std::string("cannot write ") + path);
    return GVA_OK;
}

double gva_result_gpu_ms(const gva_result* res) { return res ? res->r.gpu_ms : 0.0; }

void gva_result_free(gva_result* res) {
    if (!res) return;
    MatchResult* m = new MatchResult(std::move(res->r));
    free_result(m);
    delete res;
}

int gva_db_set_graphs(gva_db* db, const uint64_t* first, uint32_t num_graphs) {
    if (!db) return fail(GVA_ERR_ARG, "null argument");
    return set_graph_ids(*db->dev, first, num_graphs);
}

namespace {
int rounds_mode(int flags) {
    if (flags & GVA_BATCH_HOST_ROUNDS) return ROUNDS_HOST;
    if (flags & GVA_BATCH_DEVICE_ROUNDS) return ROUNDS_DEVICE;
    return ROUNDS_AUTO;
}

void fill_batch_stats(const BatchStats& bs, double lower_ms, gva_batch_stats* stats) {
    memset(stats, 0, sizeof *stats);
    stats->gpu_ms = bs.gpu_ms;
    stats->rounds = bs.rounds;
    stats->splits = bs.splits;
    stats->launches = bs.launches;
    stats->trie_nodes = bs.nodes;
    stats->lower_ms = lower_ms;
    stats->submit_ms = bs.submit_ms;
    stats->round_host_ms = bs.round_host_ms;
    stats->wait_ms = bs.wait_ms;
    stats->session_ms = bs.session_ms;
    for (int i = 0; i < 5; ++i) stats->round_phase_ms[i] = bs.phase_ms[i];
    for (int i = 0; i < 9; ++i) stats->timeline_ms[i] = bs.timeline_ms[i];
    stats->device_rounds = bs.device_rounds;
    for (int i = 0; i < K_NUM && i < 5; ++i) {
        strncpy(stats->kernels[i].name, kKernelNames[i], sizeof stats->kernels[i].name - 1);
        stats->kernels[i].launches = bs.kstat[i].launches;
        stats->kernels[i].ms = bs.kstat[i].ms;
        stats->kernels[i].bytes = bs.kstat[i].bytes;
        stats->kernels[i].rows = bs.kstat[i].rows;
    }
}
}  // namespace

int gva_batch_count(gva_db* db, const gva_plan* const* plans, int nplans, const gva_batch_opts* opts,
                    uint64_t* counts, uint64_t* graph_counts, uint32_t* graph_support, gva_batch_stats* stats) {
    if (!db || (nplans > 0 && (!plans || !counts))) return fail(GVA_ERR_ARG, "null argument");
    gva_batch_opts o{};
    if (opts) o = *opts;
    if ((o.flags & GVA_BATCH_HOST_ROUNDS) && (o.flags & GVA_BATCH_DEVICE_ROUNDS))
        return fail(GVA_ERR_ARG, "GVA_BATCH_HOST_ROUNDS and GVA_BATCH_DEVICE_ROUNDS exclude each other");
    std::vector<std::vector<Step>> steps(nplans);
    for (int i = 0; i < nplans; ++i)
        if (!plans[i]) return fail(GVA_ERR_ARG, "null plan");
    const auto t_lower = std::chrono::steady_clock::now();
    {
        int st = parallel_for(nplans, [&](int i) { return lower_plan(plans[i]->plan, db->dev->meta, steps[i], true); });
        if (st) return st;
    }
    const double lower_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_lower).count();
    BatchStats bs;
    int st = run_batch(*db->dev, std::move(steps), (cudaStream_t)o.stream, o.budget_bytes, db->dev->vgraph,
                       db->dev->num_graphs,
                       counts, graph_counts, graph_support, o.profile != 0, &bs, rounds_mode(o.flags));
    if (stats) fill_batch_stats(bs, lower_ms, stats);
    return st;
}

int gva_batch_count_texts(gva_db* db, const char* const* texts, int n, int mode, const gva_batch_opts* opts,
                          uint64_t* counts, uint64_t* graph_counts, uint32_t* graph_support, int* status,
                          gva_batch_stats* stats) {
    if (!db || n < 0 || (n > 0 && (!texts || !counts))) return fail(GVA_ERR_ARG, "null argument");
    if (mode != GVA_MODE_DV && mode != GVA_MODE_SV) return fail(GVA_ERR_ARG, "mode must be GVA_MODE_DV or GVA_MODE_SV");
    gva_batch_opts o{};
    if (opts) o = *opts;
    if ((o.flags & GVA_BATCH_HOST_ROUNDS) && (o.flags & GVA_BATCH_DEVICE_ROUNDS))
        return fail(GVA_ERR_ARG, "GVA_BATCH_HOST_ROUNDS and GVA_BATCH_DEVICE_ROUNDS exclude each other");
    const auto t_lower = std::chrono::steady_clock::now();
    std::vector<std::vector<Step>> steps(n);
    std::vector<int> st(n, GVA_OK);
    std::vector<std::string> msg(n);
    const HostGraph& meta = db->dev->meta;
    // device planning: queries read on the host, planned by the planning
    // kernel, lowered on the host from the compact plans
    const bool on_device = (o.flags & GVA_BATCH_PLAN_ON_DEVICE) && mode == GVA_MODE_DV;
    std::vector<std::vector<uint32_t>> qlab(on_device ? n : 0), qsdl(on_device ? n : 0);
    std::vector<int> dev_slot(on_device ? n : 0, -1);
    std::vector<DevPlanOut> dev_out;
    if (on_device) {
        std::vector<int> rd(n, GVA_OK);
        parallel_for(n, [&](int i) {
            rd[i] = texts[i] ? read_query_text(texts[i], qlab[i], qsdl[i]) : fail(GVA_ERR_ARG, "null query text");
            if (rd[i]) msg[i] = last_error_cstr();
            return GVA_OK;
        });
        std::vector<DevPlanQuery> dq;
        for (int i = 0; i < n; ++i) {
            const std::vector<uint32_t>& lab = qlab[i];
            const std::vector<uint32_t>& sdl = qsdl[i];
            if (rd[i]) {
                st[i] = rd[i];
                continue;
            }
            bool ok = !sdl.empty() && lab.size() <= (size_t)kDevPlanV && sdl.size() / 3 <= (size_t)kDevPlanLines;
            for (size_t e = 0; e + 2 < sdl.size() && ok; e += 3)
                ok = sdl[e] < lab.size() && sdl[e + 1] < lab.size() && sdl[e] != sdl[e + 1];
            if (!ok) continue;
            DevPlanQuery q{};
            q.n = (uint32_t)lab.size();
            q.lines = (uint32_t)(sdl.size() / 3);
            for (size_t v = 0; v < lab.size(); ++v) q.label[v] = lab[v];
            for (uint32_t e = 0; e < q.lines; ++e) {
                q.s[e] = (uint8_t)sdl[3 * e];
                q.d[e] = (uint8_t)sdl[3 * e + 1];
                q.l[e] = sdl[3 * e + 2];
            }
            dev_slot[i] = (int)dq.size();
            dq.push_back(q);
        }
        dev_out.resize(dq.size());
        const int rc = plan_on_device(db->dev->device, (cudaStream_t)o.stream, dq.data(), (uint32_t)dq.size(),
                                      dev_out.data());
        if (rc) return rc;
    }
    parallel_for(n, [&](int i) {
        thread_local std::unique_ptr<DPlanQuery> dq(new DPlanQuery());
        thread_local std::unique_ptr<DPlan> dp(new DPlan());
        if (on_device && st[i]) return GVA_OK;  // the text could not be read (message kept)
        std::vector<uint32_t> labels, sdl;
        int r = GVA_OK;
        if (on_device) {
            labels.swap(qlab[i]);
            sdl.swap(qsdl[i]);
        } else {
            r = texts[i] ? read_query_text(texts[i], labels, sdl) : fail(GVA_ERR_ARG, "null query text");
        }
        bool done = false;
        if (!r && on_device && dev_slot[i] >= 0 && dev_out[dev_slot[i]].status == DPLAN_OK) {
            dplan_from_device(dev_out[dev_slot[i]], *dp);
            r = lower_dplan(*dp, labels.data(), meta, steps[i], true);
            done = true;
        }
        if (!r && !done && !on_device && mode == GVA_MODE_DV && labels.size() <= (size_t)kDpV &&
            sdl.size() / 3 <= (size_t)kDpLines) {
            // edges the planner would reject go to it for their message
            bool clean = !sdl.empty();
            for (size_t e = 0; e + 2 < sdl.size() && clean; e += 3)
                clean = sdl[e] < labels.size() && sdl[e + 1] < labels.size() && sdl[e] != sdl[e + 1];
            if (clean) {
                dq->n = (uint32_t)labels.size();
                dq->lines = (uint32_t)(sdl.size() / 3);
                for (size_t v = 0; v < labels.size(); ++v) dq->label[v] = labels[v];
                for (uint32_t e = 0; e < dq->lines; ++e) {
                    dq->s[e] = sdl[3 * e];
                    dq->d[e] = sdl[3 * e + 1];
                    dq->l[e] = sdl[3 * e + 2];
                }
                dplan(*dq, *dp);
                if (dp->status == DPLAN_OK) {
                    r = lower_dplan(*dp, dq->label, meta, steps[i], true);
                    done = true;
                }
            }
        }
        if (!r && !done) {
            Plan plan;
            r = plan_from_query((uint32_t)labels.size(), labels.data(), sdl.data(), sdl.size() / 3, mode, plan);
            if (!r) r = lower_plan(plan, meta, steps[i], true);
        }
        st[i] = r;
        if (r) msg[i] = last_error_cstr();
        return GVA_OK;  // per-query failures are reported in status
    });
    // texts that failed to plan are counted as a plan that cannot match
    int first = -1;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (st[i] && first < 0) first = i;
        if (st[i]) {
            Step seed;
            seed.kind = STEP_SEED;
            seed.always_empty = 1;
            Step ext;
            ext.always_empty = 1;
            steps[i] = {seed, ext};
        }
    }
    const double lower_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_lower).count();
    BatchStats bs;
    int rc = n ? run_batch(*db->dev, std::move(steps), (cudaStream_t)o.stream, o.budget_bytes, db->dev->vgraph,
                           db->dev->num_graphs, counts, graph_counts, graph_support, o.profile != 0, &bs,
                           rounds_mode(o.flags))
               : GVA_OK;
    if (stats) fill_batch_stats(bs, lower_ms, stats);
    if (rc) return rc;
    if (first >= 0) return fail(st[first], "query " + std::to_string(first) + ": " + msg[first]);
    return GVA_OK;
}

int gva_db_get_tuning(const gva_db* db, gva_tuning* out) {
    if (!db || !out) return fail(GVA_ERR_ARG, "null argument");
    memset(out, 0, sizeof *out);
    out->rows_per_item = db->dev->tune_rows_per_item;
    out->hub = db->dev->tune_hub;
    const uint64_t region = db->dev->round_region_bytes.load();
    out->round_region_mb = (uint32_t)((region ? region : (2ull << 30)) >> 20);
    return GVA_OK;
}

int gva_db_set_tuning(gva_db* db, const gva_tuning* t) {
    if (!db || !t) return fail(GVA_ERR_ARG, "null argument");
    if (t->rows_per_item != 32 && t->rows_per_item != 64 && t->rows_per_item != 128)
        return fail(GVA_ERR_ARG, "rows_per_item must be 32, 64 or 128");  // hub: any value (0: every row shared)
    db->dev->tune_rows_per_item = t->rows_per_item;
    db->dev->tune_hub = t->hub;
    if (t->round_region_mb) db->dev->round_region_bytes.store((uint64_t)t->round_region_mb << 20);
    return GVA_OK;
}

int gva_db_autotune(gva_db* db, const gva_plan* const* plans, int nplans, void* stream, gva_tuning* out) {
    if (!db || nplans <= 0 || !plans) return fail(GVA_ERR_ARG, "null argument");
    std::vector<std::vector<Step>> steps(nplans);
    for (int i = 0; i < nplans; ++i)
        if (!plans[i]) return fail(GVA_ERR_ARG, "null plan");
    int st = parallel_for(nplans, [&](int i) { return lower_plan(plans[i]->plan, db->dev->meta, steps[i], true); });
    if (st) return st;
    TuneResult tr;
    st = autotune_batch(*db->dev, steps, (cudaStream_t)stream, db->dev->vgraph != nullptr, tr);
    if (st) return st;
    if (out) {
        memset(out, 0, sizeof *out);
        out->rows_per_item = tr.rows_per_item;
        out->hub = tr.hub;
        out->ms = tr.ms;
        out->default_ms = tr.default_ms;
        out->tried = (uint32_t)tr.tried.size();
    }
    return GVA_OK;
}

int gva_mine(gva_db* db, const gva_mine_opts* opts, gva_mine_result** out) {
    if (!db || !opts || !out) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    gva_mine_result* r = new gva_mine_result();
    int st = run_mine(*db->dev, (cudaStream_t)opts->stream, opts->budget_bytes, opts->max_edges, opts->min_support,
                      opts->batch_limit, opts->profile != 0, opts->reduce, opts->reduce_user, opts->support_mode,
                      opts->mni_cap, r->pats, r->stats, opts->cancel, opts->sm_percent, opts->host_threads);
    if (st) {
        delete r;
        return st;
    }
    *out = r;
    return GVA_OK;
}

int gva_mine_host(uint32_t num_labels, const uint32_t* labels, uint32_t num_edge_labels,
                  const uint8_t* has_edge_label, uint32_t max_edges, uint32_t min_support, uint32_t host_threads,
                  gva_eval_fn evaluate, void* eval_user, gva_reduce_fn reduce, void* reduce_user,
                  gva_mine_result** out) {
    if (!out || !labels || !has_edge_label) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    gva_mine_result* r = new gva_mine_result();
    std::vector<uint32_t> lab(labels, labels + num_labels);
    int st = run_mine_host(lab, num_edge_labels, has_edge_label, max_edges, min_support, host_threads, evaluate,
                           eval_user, reduce, reduce_user, r->pats, r->stats);
    if (st) {
        delete r;
        return st;
    }
    *out = r;
    return GVA_OK;
}

int gva_mine_num_patterns(const gva_mine_result* res) { return res ? (int)res->pats.size() : -1; }

int gva_mine_get(const gva_mine_result* res, int index, uint32_t* edges, uint32_t* support, uint64_t* embeddings) {
    if (!res || index < 0 || index >= (int)res->pats.size()) return fail(GVA_ERR_ARG, "pattern index out of range");
    const MinedPattern& p = res->pats[index];
    if (edges) *edges = p.edges;
    if (support) *support = p.support;
    if (embeddings) *embeddings = p.embeddings;
    return GVA_OK;
}

size_t gva_mine_pattern_text(const gva_mine_result* res, int index, char* buf, size_t cap) {
    if (!res || index < 0 || index >= (int)res->pats.size()) return 0;
    const std::string& s = res->pats[index].text;
    if (buf && cap) {
        size_t n = std::min(cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}

size_t gva_mine_export(const gva_mine_result* res, char* text_buf, size_t text_cap, uint64_t* offsets,
                       uint32_t* edges, uint32_t* supports, uint64_t* embeddings) {
    if (!res) return 0;
    size_t need = 0;
    for (const MinedPattern& p : res->pats) need += p.text.size() + 1;
    const size_t n = res->pats.size();
    for (size_t i = 0; i < n; ++i) {
        if (edges) edges[i] = res->pats[i].edges;
        if (supports) supports[i] = res->pats[i].support;
        if (embeddings) embeddings[i] = res->pats[i].embeddings;
    }
    if (text_buf && offsets && text_cap >= need) {
        size_t at = 0;
        for (size_t i = 0; i < n; ++i) {
            const std::string& t = res->pats[i].text;
            offsets[i] = at;
            memcpy(text_buf + at, t.data(), t.size());
            text_buf[at + t.size()] = 0;
            at += t.size() + 1;
        }
    }
    return need;
}

int gva_mine_get_stats(const gva_mine_result* res, gva_mine_stats* out) {
    if (!res || !out) return fail(GVA_ERR_ARG, "null argument");
    out->candidates = res->stats.candidates;
    out->frequent = res->stats.frequent;
    out->embeddings = res->stats.embeddings;
    out->levels = res->stats.levels;
    out->pruned = res->stats.pruned;
    out->gpu_ms = res->stats.gpu_ms;
    out->host_ms = res->stats.host_ms;
    out->gen_ms = res->stats.gen_ms;
    out->plan_ms = res->stats.plan_ms;
    out->eval_ms = res->stats.eval_ms;
    out->merge_ms = res->stats.merge_ms;
    out->submit_ms = res->stats.submit_ms;
    out->round_host_ms = res->stats.round_host_ms;
    out->wait_ms = res->stats.wait_ms;
    out->mni_tasks = res->stats.mni_tasks;
    out->mni_rounds = res->stats.mni_rounds;
    return GVA_OK;
}

int gva_mni_support(gva_db* db, const char* const* pattern_texts, int n, const gva_mni_opts* opts, uint32_t* support,
                    gva_mni_stats* stats) {
    if (!db || n < 0 || (n > 0 && (!pattern_texts || !support))) return fail(GVA_ERR_ARG, "null argument");
    gva_mni_opts o{};
    if (opts) o = *opts;
    std::vector<MniPattern> pats(n);
    std::vector<char> absent(n, 0);
    for (int i = 0; i < n; ++i) {
        if (!pattern_texts[i]) return fail(GVA_ERR_ARG, "null pattern text");
        bool ab = false;
        int st = mni_pattern_from_text(*db->dev, pattern_texts[i], pats[i], ab);
        if (st) return st;
        absent[i] = ab ? 1 : 0;
    }
    std::vector<uint32_t> sup;
    MniStats ms;
    int st = run_mni(*db->dev, pats, absent, o.cap, o.plain != 0, o.profile != 0, (cudaStream_t)o.stream, sup, ms);
    if (st) return st;
    for (int i = 0; i < n; ++i) support[i] = sup[i];
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->gpu_ms = ms.gpu_ms;
        stats->rounds = ms.rounds;
        stats->launches = ms.launches;
        stats->tasks = ms.tasks;
        stats->seeds = ms.seeds;
        stats->roots = ms.roots;
        stats->found = ms.found;
        strncpy(stats->kernel.name, kKernelNames[K_MNI], sizeof stats->kernel.name - 1);
        stats->kernel.launches = ms.kstat.launches;
        stats->kernel.ms = ms.kstat.ms;
        stats->kernel.bytes = ms.kstat.bytes;
        stats->kernel.rows = ms.kstat.rows;
    }
    return GVA_OK;
}

int gva_mine_kernel_stats(const gva_mine_result* res, gva_kernel_stat* out, int cap) {
    if (!res) return -1;
    for (int i = 0; i < K_NUM && i < cap; ++i) {
        memset(&out[i], 0, sizeof out[i]);
        strncpy(out[i].name, kKernelNames[i], sizeof out[i].name - 1);
        out[i].launches = res->stats.kstat[i].launches;
        out[i].ms = res->stats.kstat[i].ms;
        out[i].bytes = res->stats.kstat[i].bytes;
        out[i].rows = res->stats.kstat[i].rows;
    }
    return K_NUM;
}

void gva_mine_free(gva_mine_result* res) { delete res; }

int gva_session_create(gva_db* db, void* stream, uint64_t budget_bytes, uint32_t support_slots, gva_session** out) {
    if (!db || !out) return fail(GVA_ERR_ARG, "null argument");
    *out = nullptr;
    gva_session* h = new gva_session();
    h->db = db;
    h->ses = new BatchSession(*db->dev, (cudaStream_t)stream, budget_bytes, support_slots, false, false);
    int st = h->ses->init();
    if (st) {
        delete h->ses;
        delete h;
        return st;
    }
    *out = h;
    return GVA_OK;
}

int gva_session_submit(gva_session* s, const gva_plan* const* plans, const uint64_t* tags, int n) {
    if (!s || (n > 0 && !plans)) return fail(GVA_ERR_ARG, "null argument");
    std::vector<std::vector<Step>> steps(n);
    std::vector<uint64_t> tg(n);
    for (int i = 0; i < n; ++i) {
        if (!plans[i]) return fail(GVA_ERR_ARG, "null plan");
        int st = lower_plan(plans[i]->plan, s->db->dev->meta, steps[i], true);
        if (st) return st;
        tg[i] = tags ? tags[i] : (uint64_t)i;
    }
    return s->ses->submit(std::move(steps), tg, nullptr);
}

int gva_session_round(gva_session* s, int* active_tasks) {
    if (!s) return fail(GVA_ERR_ARG, "null argument");
    int st = s->ses->round();
    for (int q : s->ses->take_completed()) s->ready.push_back(q);
    if (active_tasks) *active_tasks = (int)s->ses->num_active();
    return st;
}

int gva_session_poll(gva_session* s, uint64_t* tags, uint64_t* counts, uint32_t* supports, int cap) {
    if (!s) return -1;
    int n = 0;
    while (n < cap && !s->ready.empty()) {
        const int q = s->ready.front();
        const auto& p = s->ses->plan(q);
        if (tags) tags[n] = p.tag;
        if (counts) counts[n] = p.count;
        uint32_t sup = 0;
        if (supports && s->ses->words() > 0 && s->ses->read_support(q, &sup, nullptr)) return -1;
        if (supports) supports[n] = sup;
        s->ses->release(q);
        s->ready.erase(s->ready.begin());
        ++n;
    }
    return n;
}

void gva_session_free(gva_session* s) {
    if (!s) return;
    delete s->ses;
    delete s;
}

int gva_plan_num_steps(const gva_plan* plan, const gva_db* db) {
    if (!plan || !db) return -1;
    std::vector<Step> s;
    if (steps_for(plan, db, s)) return -1;
    return (int)s.size();
}

int gva_plan_step_width_in(const gva_plan* plan, const gva_db* db, int step) {
    std::vector<Step> s;
    if (!plan || !db || steps_for(plan, db, s) || step < 0 || step >= (int)s.size()) return -1;
    return (int)s[step].width_in;
}

int gva_plan_step_width_out(const gva_plan* plan, const gva_db* db, int step) {
    std::vector<Step> s;
    if (!plan || !db || steps_for(plan, db, s) || step < 0 || step >= (int)s.size()) return -1;
    const Step& t = s[step];
    return t.kind == STEP_SEED ? 1 : (t.kind == STEP_EXT ? (int)t.width_in + 1 : (int)t.width_in);
}

size_t gva_step_scratch_bytes(uint64_t in_rows) { return step_scratch_bytes(in_rows); }

int gva_step_run(gva_db* db, const gva_plan* plan, int step, const uint32_t* in_dev, uint64_t in_rows,
                 uint32_t* out_dev, uint64_t out_capacity_rows, uint64_t* out_rows, void* scratch_dev,
                 size_t scratch_bytes, void* stream) {
    if (!db || !plan) return fail(GVA_ERR_ARG, "null argument");
    std::vector<Step> s;
    int st = steps_for(plan, db, s);
    if (st) return st;
    if (step < 0 || step >= (int)s.size()) return fail(GVA_ERR_ARG, "step index out of range");
    return run_step(*db->dev, s[step], in_dev, in_rows, out_dev, out_capacity_rows, out_rows, scratch_dev,
                    scratch_bytes, (cudaStream_t)stream);
}

int gva_step_run_static(gva_db* db, const gva_plan* plan, int step, const uint32_t* in_dev, uint64_t in_rows,
                        uint32_t* out_dev, uint64_t out_capacity_rows, uint64_t* out_rows, void* stream) {
    if (!db || !plan) return fail(GVA_ERR_ARG, "null argument");
    std::vector<Step> s;
    int st = steps_for(plan, db, s);
    if (st) return st;
    if (step < 0 || step >= (int)s.size()) return fail(GVA_ERR_ARG, "step index out of range");
    return run_step_static(*db->dev, s[step], in_dev, in_rows, out_dev, out_capacity_rows, out_rows,
                           (cudaStream_t)stream);
}

}  // extern "C"
