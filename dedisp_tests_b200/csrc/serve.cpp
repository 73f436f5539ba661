// Streaming dedispersion server (see serve.hpp).
#include "serve.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>

#include "dedisp_b200.h"
#include "errors.hpp"
#include "fdd/FDDGPUPlan.hpp"
#include "host_math.hpp"
#include "runtime.hpp"
#include "tdd/TDDPlan.hpp"

namespace dedisp {
namespace detail {

namespace {
double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

struct StreamServer::Beam {
    int kind = 0;
    int group = 0;               // index of the distinct (kind, DM list)
    std::vector<float> dms;
    size_t max_delay = 0;
    rt::DeviceBuffer ring[2];    // [max_delay + max_gulp] input rows each
    int cur = 0;                 // ring holding the tail in rows [0, max_delay)
    bool busy = false;
};

struct StreamServer::Worker {
    int id = 0;
    int kind = 0;
    std::unique_ptr<rt::Stream> stream;
    std::map<int, std::unique_ptr<Plan>> plans;  // by DM-list group
    rt::DeviceBuffer out;                        // ndm_max x max_gulp floats
    std::unique_ptr<rt::Event> e0, e1;
    std::thread thread;
};

StreamServer::StreamServer(const ServeConfig& cfg) : m_cfg(cfg)
{
    const int nb = cfg.in_nbits;
    if (nb != 1 && nb != 2 && nb != 4 && nb != 8 && nb != 16 && nb != 32) DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    if (cfg.nchans == 0 || (cfg.nchans * (size_t)nb) % 32 != 0) DD_THROW(DEDISP_INVALID_STRIDE);
    if (cfg.max_gulp == 0) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "max_gulp must be positive");
    if (cfg.tdd_workers < 0 || cfg.fdd_workers < 0 || cfg.tdd_workers + cfg.fdd_workers == 0)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "the server needs at least one worker");
    m_row_bytes = cfg.nchans * (size_t)nb / 8;
    if (m_cfg.fdd_max_gulp == 0 || m_cfg.fdd_max_gulp > m_cfg.max_gulp) m_cfg.fdd_max_gulp = m_cfg.max_gulp;
    m_delays.assign(cfg.nchans + 1, 0.f);
    hostmath::delay_table(cfg.nchans, cfg.dt, cfg.f0, cfg.df, m_delays.data());
}

StreamServer::~StreamServer()
{
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_stop = true;
    }
    m_cv_work.notify_all();
    for (auto& w : m_workers)
        if (w->thread.joinable()) w->thread.join();
    if (m_started) {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != m_cfg.device) cudaSetDevice(m_cfg.device);
        cudaDeviceSynchronize();
    }
}

int StreamServer::add_beam(const float* dms, size_t ndm, int kind)
{
    if (m_started) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "beams are added before start()");
    if (!dms || ndm == 0) DD_THROW(DEDISP_NO_DM_LIST_SET);
    if (kind != 0 && kind != 1) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "kind must be 0 (TDD) or 1 (FDD)");
    if (kind == 0 && m_cfg.tdd_workers == 0) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no TDD workers");
    if (kind == 1 && m_cfg.fdd_workers == 0) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no FDD workers");
    std::unique_ptr<Beam> b(new Beam);
    b->kind = kind;
    b->dms.assign(dms, dms + ndm);
    b->max_delay = hostmath::max_delay(b->dms.back(), m_delays[m_cfg.nchans - 1]);
    b->group = -1;
    for (auto& o : m_beams)
        if (o->kind == kind && o->dms == b->dms) b->group = o->group;
    if (b->group < 0) {
        int g = 0;
        for (auto& o : m_beams) g = std::max(g, o->group + 1);
        b->group = g;
    }
    m_beams.push_back(std::move(b));
    return (int)m_beams.size() - 1;
}

size_t StreamServer::max_delay(int beam) const { return m_beams.at(beam)->max_delay; }
size_t StreamServer::dm_count(int beam) const { return m_beams.at(beam)->dms.size(); }

size_t StreamServer::start()
{
    if (m_started) return m_bytes;
    if (m_beams.empty()) DD_THROW(DEDISP_NO_DM_LIST_SET);
    rt::DeviceGuard g(m_cfg.device);
    RT_CHECK(cudaDeviceSynchronize());
    size_t free0 = 0, total = 0;
    RT_CHECK(cudaMemGetInfo(&free0, &total));
    size_t ndm_max = 0, md_max = 0;
    for (auto& b : m_beams) {
        ndm_max = std::max(ndm_max, b->dms.size());
        md_max = std::max(md_max, b->max_delay);
        for (auto& r : b->ring) {
            r.reserve((b->max_delay + m_cfg.max_gulp) * m_row_bytes);
            RT_CHECK(cudaMemset(r.get(), 0, (b->max_delay + m_cfg.max_gulp) * m_row_bytes));
        }
    }
    // Workers: one plan per DM-list group of the worker's kind, sized by a
    // warm-up at the largest gulp on zero rows.
    const int nw = m_cfg.tdd_workers + m_cfg.fdd_workers;
    for (int i = 0; i < nw; ++i) {
        std::unique_ptr<Worker> w(new Worker);
        w->id = i;
        w->kind = i < m_cfg.tdd_workers ? 0 : 1;
        w->stream.reset(new rt::Stream());
        w->e0.reset(new rt::Event(true));
        w->e1.reset(new rt::Event(true));
        w->out.reserve(ndm_max * m_cfg.max_gulp * sizeof(float));
        for (auto& b : m_beams) {
            if (b->kind != w->kind || w->plans.count(b->group)) continue;
            std::unique_ptr<Plan> p;
            if (w->kind == 0) {
                auto* t = new TDDPlan(m_cfg.nchans, m_cfg.dt, m_cfg.f0, m_cfg.df, m_cfg.device);
                p.reset(t);
            } else {
                auto* f = new FDDGPUPlan(m_cfg.nchans, m_cfg.dt, m_cfg.f0, m_cfg.df, m_cfg.device);
                FddOptions o;
                o.segmented = 1;
                o.output = FddOutput::TimeSeries;
                o.precision = m_cfg.fdd_precision ? FddPrecision::BF16x3 : FddPrecision::FP32;
                o.segment_nfft = m_cfg.fdd_segment;
                f->set_options(o);
                p.reset(f);
            }
            p->set_dm_list(b->dms.data(), b->dms.size());
            dynamic_cast<GPUPlan*>(p.get())->set_stream(w->stream->get());
            const size_t ns = b->max_delay + (w->kind == 0 ? m_cfg.max_gulp : m_cfg.fdd_max_gulp);
            p->execute(ns, b->ring[0].get<uint8_t>(), m_cfg.in_nbits, w->out.get<uint8_t>(), 32,
                       DEDISP_DEVICE_POINTERS);
            RT_CHECK(cudaStreamSynchronize(w->stream->get()));
            w->plans[b->group] = std::move(p);
        }
        m_workers.push_back(std::move(w));
    }
    RT_CHECK(cudaDeviceSynchronize());
    size_t free1 = 0;
    RT_CHECK(cudaMemGetInfo(&free1, &total));
    m_bytes = free0 > free1 ? free0 - free1 : 0;
    if (m_cfg.hbm_budget && m_bytes > m_cfg.hbm_budget)
        DD_THROW_MSG(DEDISP_MEM_ALLOC_FAILED, ("server needs " + std::to_string(m_bytes) +
                                               " device bytes, above the budget").c_str());
    m_started = true;
    for (auto& w : m_workers) {
        Worker* wp = w.get();
        w->thread = std::thread([this, wp] { worker_loop(wp); });
    }
    return m_bytes;
}

long StreamServer::submit(int beam, const uint8_t* rows, size_t n, float* d_out)
{
    if (!m_started) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "submit before start()");
    if (beam < 0 || beam >= (int)m_beams.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no such beam");
    if (!rows) DD_THROW(DEDISP_INVALID_POINTER);
    if (n == 0 || n > m_cfg.max_gulp) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "gulp length outside 1..max_gulp");
    if (m_beams[beam]->kind == 1 && n > m_cfg.fdd_max_gulp)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "FDD gulp longer than fdd_max_gulp");
    std::lock_guard<std::mutex> lk(m_mu);
    if (!m_error.empty()) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, m_error.c_str());
    const long t = (long)m_records.size();
    GulpRecord r;
    r.beam = beam;
    r.nsamps = n;
    r.t_submit = now_s();
    m_records.push_back(r);
    m_done.push_back(0);
    m_queue.push_back(Job{t, beam, rows, n, d_out, r.t_submit});
    m_cv_work.notify_all();
    return t;
}

void StreamServer::worker_loop(Worker* w)
{
    try {
        rt::DeviceGuard g(m_cfg.device);
        for (;;) {
            Job job{-1, -1, nullptr, 0, nullptr, 0.0};
            {
                std::unique_lock<std::mutex> lk(m_mu);
                auto pick = [&]() -> bool {
                    for (auto it = m_queue.begin(); it != m_queue.end(); ++it) {
                        Beam& b = *m_beams[it->beam];
                        if (b.kind != w->kind) continue;
                        if (b.busy) continue;
                        // earlier queued gulps of the same beam go first
                        bool earlier = false;
                        for (auto jt = m_queue.begin(); jt != it; ++jt)
                            if (jt->beam == it->beam) earlier = true;
                        if (earlier) continue;
                        job = *it;
                        m_queue.erase(it);
                        b.busy = true;
                        return true;
                    }
                    return false;
                };
                m_cv_work.wait(lk, [&] { return m_stop || pick(); });
                if (job.beam < 0) return;  // stopping
            }
            GulpRecord rec;
            run_job(w, job, rec);
            {
                std::lock_guard<std::mutex> lk(m_mu);
                GulpRecord& r = m_records[job.ticket];
                r.t_start = rec.t_start;
                r.t_done = rec.t_done;
                r.device_ms = rec.device_ms;
                r.worker = w->id;
                m_done[job.ticket] = 1;
                m_beams[job.beam]->busy = false;
            }
            m_cv_done.notify_all();
            m_cv_work.notify_all();
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(m_mu);
        m_error = e.what();
        m_stop = true;
        m_cv_done.notify_all();
        m_cv_work.notify_all();
    }
}

void StreamServer::run_job(Worker* w, const Job& j, GulpRecord& rec)
{
    Beam& b = *m_beams[j.beam];
    cudaStream_t s = w->stream->get();
    rec.t_start = now_s();
    uint8_t* ring = b.ring[b.cur].get<uint8_t>();
    uint8_t* next = b.ring[1 - b.cur].get<uint8_t>();
    const size_t md = b.max_delay;
    float* out = j.d_out ? j.d_out : w->out.get<float>();
    w->e0->record(s);
    RT_CHECK(cudaMemcpyAsync(ring + md * m_row_bytes, j.rows, j.n * m_row_bytes, cudaMemcpyHostToDevice, s));
    Plan& p = *w->plans.at(b.group);
    p.execute(md + j.n, ring, m_cfg.in_nbits, reinterpret_cast<uint8_t*>(out), 32,
              DEDISP_DEVICE_POINTERS | (w->kind == 0 ? DEDISP_ASYNC : 0));
    // the last max_delay rows become the next gulp's tail
    if (md) RT_CHECK(cudaMemcpyAsync(next, ring + j.n * m_row_bytes, md * m_row_bytes, cudaMemcpyDeviceToDevice, s));
    w->e1->record(s);
    RT_CHECK(cudaStreamSynchronize(s));
    b.cur = 1 - b.cur;
    rec.t_done = now_s();
    RT_CHECK(cudaEventElapsedTime(&rec.device_ms, w->e0->get(), w->e1->get()));
}

bool StreamServer::done(long ticket)
{
    std::lock_guard<std::mutex> lk(m_mu);
    if (ticket < 0 || ticket >= (long)m_done.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no such ticket");
    if (!m_error.empty()) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, m_error.c_str());
    return m_done[ticket] != 0;
}

void StreamServer::wait(long ticket)
{
    std::unique_lock<std::mutex> lk(m_mu);
    if (ticket < 0 || ticket >= (long)m_done.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no such ticket");
    m_cv_done.wait(lk, [&] { return m_done[ticket] != 0 || !m_error.empty(); });
    if (!m_error.empty()) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, m_error.c_str());
}

void StreamServer::drain()
{
    std::unique_lock<std::mutex> lk(m_mu);
    m_cv_done.wait(lk, [&] {
        if (!m_error.empty()) return true;
        return std::all_of(m_done.begin(), m_done.end(), [](char d) { return d != 0; });
    });
    if (!m_error.empty()) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, m_error.c_str());
}

std::vector<GulpRecord> StreamServer::records() const
{
    std::lock_guard<std::mutex> lk(m_mu);
    return m_records;
}

}  // namespace detail
}  // namespace dedisp

// ---------------------------------------------------------------------------
// C interface (include/dedisp_b200.h).
// ---------------------------------------------------------------------------
struct dedisp_b200_server_struct {
    std::unique_ptr<dedisp::detail::StreamServer> s;
};

namespace dedisp {
void note_last_error(dedisp_error code, const char* msg);
}

namespace {
template <typename F>
dedisp_error server_call(dedisp_b200_server srv, F&& fn)
{
    if (!srv || !srv->s) return DEDISP_INVALID_PLAN;
    try {
        fn(*srv->s);
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        dedisp::note_last_error(e.code(), e.what());
        return e.code();
    } catch (const std::exception& e) {
        dedisp::note_last_error(DEDISP_UNKNOWN_ERROR, e.what());
        return DEDISP_UNKNOWN_ERROR;
    } catch (...) {
        return DEDISP_UNKNOWN_ERROR;
    }
}
}  // namespace

extern "C" {

dedisp_error dedisp_b200_server_create(dedisp_b200_server* server, dedisp_size nchans, dedisp_float dt,
                                       dedisp_float f0, dedisp_float df, dedisp_size in_nbits, int device,
                                       dedisp_size hbm_budget, dedisp_size max_gulp, int tdd_workers,
                                       int fdd_workers, int fdd_precision, dedisp_size fdd_segment,
                                       dedisp_size fdd_max_gulp)
{
    if (!server) return DEDISP_INVALID_POINTER;
    *server = nullptr;
    try {
        dedisp::detail::ServeConfig c;
        c.nchans = nchans;
        c.dt = dt;
        c.f0 = f0;
        c.df = df;
        c.in_nbits = (int)in_nbits;
        c.device = device;
        c.hbm_budget = hbm_budget;
        c.max_gulp = max_gulp;
        c.tdd_workers = tdd_workers;
        c.fdd_workers = fdd_workers;
        c.fdd_precision = fdd_precision;
        c.fdd_segment = fdd_segment;
        c.fdd_max_gulp = fdd_max_gulp;
        std::unique_ptr<dedisp_b200_server_struct> h(new dedisp_b200_server_struct);
        h->s.reset(new dedisp::detail::StreamServer(c));
        *server = h.release();
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        dedisp::note_last_error(e.code(), e.what());
        return e.code();
    } catch (...) {
        return DEDISP_UNKNOWN_ERROR;
    }
}

void dedisp_b200_server_destroy(dedisp_b200_server server)
{
    try {
        delete server;
    } catch (...) {
    }
}

int dedisp_b200_server_add_beam(dedisp_b200_server server, const dedisp_float* dm_list, dedisp_size dm_count,
                                int kind)
{
    int id = -1;
    if (server_call(server, [&](dedisp::detail::StreamServer& s) { id = s.add_beam(dm_list, dm_count, kind); }) !=
        DEDISP_NO_ERROR)
        return -1;
    return id;
}

dedisp_size dedisp_b200_server_max_delay(dedisp_b200_server server, int beam)
{
    dedisp_size n = 0;
    if (server_call(server, [&](dedisp::detail::StreamServer& s) { n = s.max_delay(beam); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

dedisp_error dedisp_b200_server_start(dedisp_b200_server server, dedisp_size* bytes_held)
{
    return server_call(server, [&](dedisp::detail::StreamServer& s) {
        const size_t b = s.start();
        if (bytes_held) *bytes_held = b;
    });
}

long dedisp_b200_server_submit(dedisp_b200_server server, int beam, const dedisp_byte* rows, dedisp_size nsamps,
                               dedisp_float* d_out)
{
    long t = -1;
    if (server_call(server, [&](dedisp::detail::StreamServer& s) { t = s.submit(beam, rows, nsamps, d_out); }) !=
        DEDISP_NO_ERROR)
        return -1;
    return t;
}

int dedisp_b200_server_done(dedisp_b200_server server, long ticket)
{
    int d = -1;
    if (server_call(server, [&](dedisp::detail::StreamServer& s) { d = s.done(ticket) ? 1 : 0; }) !=
        DEDISP_NO_ERROR)
        return -1;
    return d;
}

dedisp_error dedisp_b200_server_wait(dedisp_b200_server server, long ticket)
{
    return server_call(server, [&](dedisp::detail::StreamServer& s) { s.wait(ticket); });
}

dedisp_error dedisp_b200_server_drain(dedisp_b200_server server)
{
    return server_call(server, [&](dedisp::detail::StreamServer& s) { s.drain(); });
}

dedisp_size dedisp_b200_server_record_count(dedisp_b200_server server)
{
    dedisp_size n = 0;
    if (server_call(server, [&](dedisp::detail::StreamServer& s) { n = s.records().size(); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

dedisp_error dedisp_b200_server_records(dedisp_b200_server server, dedisp_b200_gulp_record* out, dedisp_size n)
{
    if (n && !out) return DEDISP_INVALID_POINTER;
    return server_call(server, [&](dedisp::detail::StreamServer& s) {
        const auto r = s.records();
        for (size_t i = 0; i < n && i < r.size(); ++i) {
            out[i].beam = r[i].beam;
            out[i].worker = r[i].worker;
            out[i].nsamps = r[i].nsamps;
            out[i].t_submit = r[i].t_submit;
            out[i].t_start = r[i].t_start;
            out[i].t_done = r[i].t_done;
            out[i].device_ms = r[i].device_ms;
        }
    });
}

}  // extern "C"
