// Serving loop: solves submitted while others run, admitted by device-memory
// footprint, each on its own CUDA stream so that their kernels overlap on the
// GPU, retired (slot and memory freed) as soon as they converge. No reference
// counterpart: the reference runs one ITPSystem per process
// (itp2d.cpp:62-135), and a request here is one such system
// (itpsystem.cpp:407-470) run to is_finished().
//
// Scheduling: continuous batching at solve granularity. Up to max_active
// worker threads each take the oldest queued request whose footprint
// (itp2d_ctx_footprint: the k states of N x N points in two or three buffers,
// plus matrices and tables) fits in the unused part of the memory budget,
// build its ITPSystem on a stream of its own, step it until it finishes and
// free it. A request larger than the whole budget is refused at submission.
// Requests keep their order when they fit; a smaller one may start before an
// older one that is waiting for memory (first fit), so one large request
// does not hold back the queue behind it.
#include "itp2d_host.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

namespace itp2d {

inline double wall_s() {
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
	long long id = 0;
	Parameters params;
	long long footprint = 0;
	double t_submit = 0, t_start = 0, t_finish = 0;
	bool done = false;
	int status = ITP2D_OK;
	int error_flag = 0, iterations = 0, converged = 0;
	std::vector<double> E, sigma;
	std::string error;
};

class Server {
  public:
	Server(int max_active, long long budget) : budget(budget) {
		for (int i = 0; i < max_active; i++) workers.emplace_back([this] { work(); });
	}
	~Server() {
		{
			std::lock_guard<std::mutex> g(mu);
			stopping = true;
		}
		cv.notify_all();
		for (auto& t : workers) t.join();
	}

	int submit(const itp2d_parameters& p, const double* extra, const double* init, long long* id) {
		const long long fp = itp2d_ctx_footprint(p.sx, p.sy, p.num_states, p.boundary, p.B, p.halforder);
		if (fp < 0) return ITP2D_E_INVALID;
		if (fp > budget) return ITP2D_E_OOM;
		auto r = std::make_shared<Request>();
		r->params.raw() = p;
		const size_t G = (size_t)p.sx * (size_t)p.sy;
		if (extra) r->params.user_potential.assign(extra, extra + G);
		if (init) r->params.initial_states.assign(init, init + 2 * G * (size_t)p.num_states);
		r->footprint = fp;
		{
			std::lock_guard<std::mutex> g(mu);
			if (stopping) return ITP2D_E_INVALID;
			r->id = ++last_id;
			r->t_submit = wall_s();
			all[r->id] = r;
			queue.push_back(r);
		}
		cv.notify_all();
		*id = r->id;
		return ITP2D_OK;
	}

	// ITP2D_E_TIMEOUT when the request has not finished within timeout_s.
	int wait(long long id, double timeout_s, itp2d_request_info* info, double* E, double* sigma) {
		std::unique_lock<std::mutex> lk(mu);
		auto it = all.find(id);
		if (it == all.end()) return ITP2D_E_INVALID;
		std::shared_ptr<Request> r = it->second;
		const auto until = std::chrono::steady_clock::now() +
				std::chrono::duration_cast<std::chrono::steady_clock::duration>(
						std::chrono::duration<double>(std::max(0.0, timeout_s)));
		if (!done_cv.wait_until(lk, until, [&] { return r->done; })) return ITP2D_E_TIMEOUT;
		if (info) {
			info->status = r->status;
			info->error_flag = r->error_flag;
			info->iterations = r->iterations;
			info->converged = r->converged;
			info->num_energies = (int)r->E.size();
			info->t_submit = r->t_submit;
			info->t_start = r->t_start;
			info->t_finish = r->t_finish;
			info->footprint_bytes = (double)r->footprint;
		}
		if (E) std::copy(r->E.begin(), r->E.end(), E);
		if (sigma) std::copy(r->sigma.begin(), r->sigma.end(), sigma);
		return ITP2D_OK;
	}

	void forget(long long id) {
		std::lock_guard<std::mutex> g(mu);
		auto it = all.find(id);
		if (it != all.end() && it->second->done) all.erase(it);
	}

	void stats(itp2d_server_stats* s) {
		std::lock_guard<std::mutex> g(mu);
		s->queued = (int)queue.size();
		s->running = running;
		s->peak_running = peak_running;
		s->completed = completed;
		s->bytes_in_use = (double)in_use;
		s->peak_bytes_in_use = (double)peak_in_use;
		s->budget_bytes = (double)budget;
		s->overlap_seconds = overlap_s;
		s->busy_seconds = busy_s;
	}

	const std::string& last_error() {
		std::lock_guard<std::mutex> g(mu);
		return error_text;
	}

  private:
	// oldest queued request that fits the unused budget (first fit)
	std::shared_ptr<Request> admit() {
		std::unique_lock<std::mutex> lk(mu);
		for (;;) {
			for (auto it = queue.begin(); it != queue.end(); ++it) {
				if (in_use + (*it)->footprint <= budget) {
					std::shared_ptr<Request> r = *it;
					queue.erase(it);
					account(+1);
					in_use += r->footprint;
					peak_in_use = std::max(peak_in_use, in_use);
					return r;
				}
			}
			// on shutdown the queue still drains: every queued request fits
			// once the running ones free their memory
			if (stopping && queue.empty()) return nullptr;
			cv.wait(lk);
		}
	}

	// running-count bookkeeping with the time integrals of "at least one" and
	// "at least two" solves running (the latter is time the solves overlapped)
	void account(int delta) {
		const double t = wall_s();
		if (running >= 1) busy_s += t - t_mark;
		if (running >= 2) overlap_s += t - t_mark;
		t_mark = t;
		running += delta;
		peak_running = std::max(peak_running, running);
	}

	void work() {
		for (;;) {
			std::shared_ptr<Request> r = admit();
			if (!r) return;
			run(*r);
			{
				std::lock_guard<std::mutex> g(mu);
				in_use -= r->footprint;
				account(-1);
				completed++;
				r->done = true;
			}
			done_cv.notify_all();
			cv.notify_all();  // memory freed: queued requests may fit now
		}
	}

	void run(Request& r) {
		r.t_start = wall_s();
		try {
			ITPSystem sys(r.params);  // a stream of its own
			while (!sys.is_finished()) sys.step();
			r.error_flag = sys.get_error_flag() ? 1 : 0;
			if (r.error_flag) r.error = sys.last_error();
			r.iterations = sys.get_total_step_counter();
			r.converged = (int)sys.how_many_finally_converged();
			const size_t k = (size_t)r.params.raw().num_states;
			r.E.resize(k);
			r.sigma.resize(k);
			for (size_t n = 0; n < k && r.iterations > 0; n++) {
				r.E[n] = sys.get_sorted_energy(n);
				r.sigma[n] = sys.get_sorted_deviation(n);
			}
		} catch (DeviceError& e) {
			r.status = e.status;
			r.error = e.what();
		} catch (std::exception& e) {
			r.status = ITP2D_E_INVALID;
			r.error = e.what();
		}
		r.t_finish = wall_s();
		if (r.status != ITP2D_OK || r.error_flag) {
			std::lock_guard<std::mutex> g(mu);
			error_text = r.error;
		}
	}

	const long long budget;
	std::mutex mu;
	std::condition_variable cv, done_cv;
	std::deque<std::shared_ptr<Request>> queue;
	std::map<long long, std::shared_ptr<Request>> all;
	std::vector<std::thread> workers;
	bool stopping = false;
	long long last_id = 0, in_use = 0, peak_in_use = 0;
	int running = 0, peak_running = 0, completed = 0;
	double t_mark = 0, busy_s = 0, overlap_s = 0;
	std::string error_text;
};

}  // namespace itp2d

struct itp2d_server {
	itp2d::Server* s = nullptr;
};

extern "C" {

int itp2d_server_create(int max_active, double memory_budget_bytes, itp2d_server** out) {
	if (!out || max_active < 1 || max_active > 64 || !(memory_budget_bytes > 0)) return ITP2D_E_INVALID;
	*out = nullptr;
	try {
		itp2d_server* h = new itp2d_server();
		h->s = new itp2d::Server(max_active, (long long)memory_budget_bytes);
		*out = h;
	} catch (std::exception&) {
		return ITP2D_E_OOM;
	}
	return ITP2D_OK;
}

int itp2d_server_submit(itp2d_server* h, const itp2d_parameters* p, const double* extra_potential,
		const double* init_states, long long* id) {
	if (!h || !p || !id) return ITP2D_E_INVALID;
	return h->s->submit(*p, extra_potential, init_states, id);
}

int itp2d_server_wait(itp2d_server* h, long long id, double timeout_s, itp2d_request_info* info, double* E,
		double* sigma) {
	if (!h) return ITP2D_E_INVALID;
	return h->s->wait(id, timeout_s, info, E, sigma);
}

int itp2d_server_forget(itp2d_server* h, long long id) {
	if (!h) return ITP2D_E_INVALID;
	h->s->forget(id);
	return ITP2D_OK;
}

int itp2d_server_get_stats(itp2d_server* h, itp2d_server_stats* st) {
	if (!h || !st) return ITP2D_E_INVALID;
	h->s->stats(st);
	return ITP2D_OK;
}

const char* itp2d_server_last_error(itp2d_server* h) { return h ? h->s->last_error().c_str() : ""; }

int itp2d_server_destroy(itp2d_server* h) {
	if (!h) return ITP2D_E_INVALID;
	delete h->s;  // finishes the queued and running requests first
	delete h;
	return ITP2D_OK;
}

}  // extern "C"

// ---- Batched form: many independent solves stepped together ----
//
// Each instance is an ITPSystem (its own context and stream); an iteration of
// the batch runs every unfinished instance's step through the batched device
// calls: the propagations (all streams), ONE launch for every instance's
// overlap eigenproblem between the overlaps and the rotations, and the
// energies; then each instance's own convergence tests and time-step schedule
// (itpsystem.cpp:407-470). Finished instances leave the batch.

struct itp2d_batch {
	std::vector<std::unique_ptr<itp2d::ITPSystem>> sys;
	std::vector<double> t_finish;
	long long iterations = 0;
	double t_start = 0, seconds = 0;
	std::string err;
};

extern "C" {

int itp2d_batch_create(int count, const itp2d_parameters* params, const double* const* extra_potentials,
		const double* const* init_states, itp2d_batch** out) {
	if (!out || count < 1 || !params) return ITP2D_E_INVALID;
	*out = nullptr;
	itp2d_batch* b = new itp2d_batch();
	try {
		for (int i = 0; i < count; i++) {
			const itp2d_parameters& p = params[i];
			itp2d::Parameters P;
			P.raw() = p;
			const size_t G = (size_t)p.sx * (size_t)p.sy;
			if (extra_potentials && extra_potentials[i])
				P.user_potential.assign(extra_potentials[i], extra_potentials[i] + G);
			if (init_states && init_states[i])
				P.initial_states.assign(init_states[i], init_states[i] + 2 * G * (size_t)p.num_states);
			if (p.num_states < 2) throw itp2d::GeneralError("batched instances need at least two states");
			b->sys.emplace_back(new itp2d::ITPSystem(P));
		}
	} catch (itp2d::DeviceError& e) {
		const int st = e.status;
		delete b;
		return st;
	} catch (std::exception&) {
		delete b;
		return ITP2D_E_INVALID;
	}
	b->t_finish.assign(count, 0.0);
	*out = b;
	return ITP2D_OK;
}

int itp2d_batch_run(itp2d_batch* b, int max_iterations) {
	if (!b) return ITP2D_E_INVALID;
	const double t0 = itp2d::wall_s();
	if (b->iterations == 0) b->t_start = t0;
	try {
		for (int it = 0; it < max_iterations; it++) {
			std::vector<itp2d::ITPSystem*> act;
			for (auto& s : b->sys)
				if (s->step_begin()) act.push_back(s.get());
			if (act.empty()) break;
			const int n = (int)act.size();
			std::vector<itp2d_ctx*> ctxs(n);
			for (int i = 0; i < n; i++) ctxs[i] = act[i]->context();
			int st = itp2d_batch_propagate(n, ctxs.data());
			if (st) throw itp2d::DeviceError("itp2d_batch_propagate", st);
			std::vector<int> ost(n), bi(n);
			std::vector<double> bv(n);
			st = itp2d_batch_orthonormalize(n, ctxs.data(), ost.data(), bi.data(), bv.data());
			if (st) throw itp2d::DeviceError("itp2d_batch_orthonormalize", st);
			for (int i = 0; i < n; i++) act[i]->orthonormalized(ost[i], bi[i], bv[i]);
			std::vector<std::vector<double>> E(n), S(n), R(n);
			std::vector<double*> pe(n), ps(n), pr(n);
			for (int i = 0; i < n; i++) {
				const size_t k = (size_t)act[i]->p.num_states;
				E[i].resize(k);
				S[i].resize(k);
				R[i].resize(k);
				pe[i] = E[i].data();
				ps[i] = S[i].data();
				pr[i] = R[i].data();
			}
			st = itp2d_batch_energies(n, ctxs.data(), pe.data(), ps.data(), pr.data());
			if (st) throw itp2d::DeviceError("itp2d_batch_energies", st);
			const double now = itp2d::wall_s();
			for (int i = 0; i < n; i++) {
				act[i]->energies_computed(pe[i], ps[i], pr[i]);
				if (act[i]->is_finished())
					for (size_t j = 0; j < b->sys.size(); j++)
						if (b->sys[j].get() == act[i]) b->t_finish[j] = now - b->t_start;
			}
			b->iterations++;
		}
	} catch (itp2d::DeviceError& e) {
		b->err = e.what();
		return e.status;
	} catch (std::exception& e) {
		b->err = e.what();
		return ITP2D_E_INVALID;
	}
	b->seconds += itp2d::wall_s() - t0;
	return ITP2D_OK;
}

int itp2d_batch_result(itp2d_batch* b, int i, itp2d_request_info* info, double* E, double* sigma) {
	if (!b || i < 0 || i >= (int)b->sys.size()) return ITP2D_E_INVALID;
	itp2d::ITPSystem& s = *b->sys[i];
	const int k = s.p.num_states;
	const bool have = s.get_total_step_counter() > 0 && !s.get_energies().empty();
	if (info) {
		std::memset(info, 0, sizeof(*info));
		info->status = ITP2D_OK;
		info->error_flag = s.get_error_flag() ? 1 : 0;
		info->iterations = s.get_total_step_counter();
		info->converged = (int)s.how_many_finally_converged();
		info->num_energies = have ? k : 0;
		info->t_finish = b->t_finish[i];
		info->footprint_bytes = (double)itp2d_ctx_device_bytes(s.context());
	}
	for (int n = 0; have && n < k; n++) {
		if (E) E[n] = s.get_sorted_energy(n);
		if (sigma) sigma[n] = s.get_sorted_deviation(n);
	}
	return ITP2D_OK;
}

int itp2d_batch_size(const itp2d_batch* b) { return b ? (int)b->sys.size() : -1; }

int itp2d_batch_finished(const itp2d_batch* b) {
	if (!b) return -1;
	for (auto& s : b->sys)
		if (!s->is_finished()) return 0;
	return 1;
}

int itp2d_batch_stats(const itp2d_batch* b, long long* iterations, double* seconds) {
	if (!b) return ITP2D_E_INVALID;
	if (iterations) *iterations = b->iterations;
	if (seconds) *seconds = b->seconds;
	return ITP2D_OK;
}

const char* itp2d_batch_last_error(const itp2d_batch* b) { return b ? b->err.c_str() : ""; }

int itp2d_batch_destroy(itp2d_batch* b) {
	if (!b) return ITP2D_E_INVALID;
	delete b;
	return ITP2D_OK;
}

}  // extern "C"
