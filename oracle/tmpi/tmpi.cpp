// tmpi.cpp -- the thread-rank runtime behind oracle/tmpi/mpi.h and the
// process entry point that starts the ranks.
//
// TEST INFRASTRUCTURE ONLY (see mpi.h): the reference's main() is compiled
// as hplai_rank_main and run by TMPI_NP threads (default 4) of this
// process; MPI calls map onto shared-memory mailboxes and collective slots.
// With TMPI_XDUMP=<file> the solution vector the reference's refinement
// returns is written there as n little-endian doubles (the reference itself
// never prints x; ref_xdump.cpp collects it).
#include "mpi.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unistd.h>
#include <vector>

extern int hplai_rank_main(int argc, char **argv);

namespace {

struct Comm {
	std::vector<int> members;   // world ranks, in comm-rank order
};

struct Message {
	int comm, src, tag;         // src: comm rank of the sender
	std::vector<char> data;
};

struct tmpi_request_base {};

}  // namespace

struct tmpi_request {
	enum Kind { DONE, RECV, BCAST } kind = DONE;
	bool done = false;
	void *buf = nullptr;
	size_t bytes = 0;
	int comm = 0, src = 0, tag = 0;
	long seq = 0;               // BCAST: collective sequence number on comm
	int root = 0;
};

namespace {

struct Mailbox {
	std::mutex mu;
	std::condition_variable cv;
	std::deque<Message> unexpected;
	std::deque<tmpi_request *> posted;
};

struct Slot {
	// Ibcast: data from the root, readers left; Allreduce / Barrier / split:
	// contributions and the result
	std::vector<char> data;
	int readers_left = 0;
	int arrived = 0;
	bool ready = false;
	std::vector<std::vector<char>> contrib;
	std::vector<std::pair<int, int>> split;   // (color, key) per comm rank
	std::vector<int> newcomm;                 // per comm rank
};

std::mutex g_mu;                 // comms, slots, sequence counters
std::condition_variable g_cv;
std::vector<Comm> g_comms;
std::map<std::pair<int, long>, Slot> g_slots;
std::map<std::pair<int, int>, long> g_seq;   // (comm, world rank) -> next collective number
std::vector<std::unique_ptr<Mailbox>> g_box;
int g_world = 1;
thread_local int t_rank = 0;

std::mutex g_x_mu;
std::vector<double> g_x;
int g_x_done = 0;
std::vector<float> g_lu;
int g_lu_done = 0;

size_t type_size(MPI_Datatype t)
{
	switch (t) {
	case MPI_BYTE: case MPI_CHAR: return 1;
	case MPI_SHORT: return 2;
	case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
	case MPI_DOUBLE: case MPI_INT64_T: case MPI_UINT64_T: case MPI_LONG_LONG: return 8;
	default:
		std::fprintf(stderr, "tmpi: unsupported datatype %d\n", t);
		std::abort();
	}
}

int comm_rank_of(int comm, int world_rank)
{
	const auto &m = g_comms.at(comm).members;
	auto it = std::find(m.begin(), m.end(), world_rank);
	return it == m.end() ? -1 : static_cast<int>(it - m.begin());
}

int my_comm_rank(int comm)
{
	std::lock_guard<std::mutex> lk(g_mu);
	return comm_rank_of(comm, t_rank);
}

int comm_size(int comm)
{
	std::lock_guard<std::mutex> lk(g_mu);
	return static_cast<int>(g_comms.at(comm).members.size());
}

int world_of(int comm, int r)
{
	std::lock_guard<std::mutex> lk(g_mu);
	return g_comms.at(comm).members.at(r);
}

long next_seq(int comm)
{
	std::lock_guard<std::mutex> lk(g_mu);
	return g_seq[{comm, t_rank}]++;
}

// Completes a receive from a message (caller holds the mailbox lock).
void fill_recv(tmpi_request *r, const Message &m)
{
	const size_t n = std::min(r->bytes, m.data.size());
	if (m.data.size() > r->bytes) {
		std::fprintf(stderr, "tmpi: message of %zu bytes truncated to %zu\n", m.data.size(), r->bytes);
		std::abort();
	}
	if (n) std::memcpy(r->buf, m.data.data(), n);
	r->done = true;
}

void deliver(int comm, int dest, int tag, const void *buf, size_t bytes)
{
	Message m;
	m.comm = comm;
	m.src = my_comm_rank(comm);
	m.tag = tag;
	Mailbox &box = *g_box.at(world_of(comm, dest));
	std::lock_guard<std::mutex> lk(box.mu);
	for (auto it = box.posted.begin(); it != box.posted.end(); ++it) {
		tmpi_request *r = *it;
		if (r->comm == comm && r->src == m.src && r->tag == tag) {
			m.data.assign(static_cast<const char *>(buf), static_cast<const char *>(buf) + bytes);
			fill_recv(r, m);
			box.posted.erase(it);
			box.cv.notify_all();
			return;
		}
	}
	m.data.assign(static_cast<const char *>(buf), static_cast<const char *>(buf) + bytes);
	box.unexpected.push_back(std::move(m));
	box.cv.notify_all();
}

// Ibcast completion on a non-root rank; true when the data was copied.
bool try_bcast(tmpi_request *r)
{
	std::lock_guard<std::mutex> lk(g_mu);
	auto it = g_slots.find({r->comm, r->seq});
	if (it == g_slots.end() || !it->second.ready) return false;
	if (r->bytes) std::memcpy(r->buf, it->second.data.data(), std::min(r->bytes, it->second.data.size()));
	r->done = true;
	if (--it->second.readers_left == 0) g_slots.erase(it);
	return true;
}

bool progress(tmpi_request *r)
{
	if (!r || r->done) return true;
	if (r->kind == tmpi_request::BCAST) return try_bcast(r);
	if (r->kind == tmpi_request::RECV) {
		Mailbox &box = *g_box.at(t_rank);
		std::lock_guard<std::mutex> lk(box.mu);
		return r->done;
	}
	return true;
}

void wait_one(tmpi_request *r)
{
	if (!r) return;
	if (r->kind == tmpi_request::RECV) {
		Mailbox &box = *g_box.at(t_rank);
		std::unique_lock<std::mutex> lk(box.mu);
		box.cv.wait(lk, [&] { return r->done; });
		return;
	}
	if (r->kind == tmpi_request::BCAST) {
		std::unique_lock<std::mutex> lk(g_mu);
		for (;;) {
			auto it = g_slots.find({r->comm, r->seq});
			if (it != g_slots.end() && it->second.ready) {
				if (r->bytes) std::memcpy(r->buf, it->second.data.data(), std::min(r->bytes, it->second.data.size()));
				r->done = true;
				if (--it->second.readers_left == 0) g_slots.erase(it);
				return;
			}
			g_cv.wait(lk);
		}
	}
}

void set_status(MPI_Status *s)
{
	if (s) *s = MPI_Status{0, 0, MPI_SUCCESS};
}

template <typename T>
void reduce_into(std::vector<char> &acc, const std::vector<char> &v, MPI_Op op)
{
	T *a = reinterpret_cast<T *>(acc.data());
	const T *b = reinterpret_cast<const T *>(v.data());
	const size_t n = acc.size() / sizeof(T);
	for (size_t i = 0; i < n; ++i) {
		if (op == MPI_SUM) a[i] = a[i] + b[i];
		else if (op == MPI_MAX) a[i] = a[i] < b[i] ? b[i] : a[i];
		else if (op == MPI_MIN) a[i] = b[i] < a[i] ? b[i] : a[i];
		else {
			std::fprintf(stderr, "tmpi: unsupported op %d\n", op);
			std::abort();
		}
	}
}

void reduce_typed(std::vector<char> &acc, const std::vector<char> &v, MPI_Datatype t, MPI_Op op)
{
	switch (t) {
	case MPI_FLOAT: reduce_into<float>(acc, v, op); break;
	case MPI_DOUBLE: reduce_into<double>(acc, v, op); break;
	case MPI_INT: reduce_into<int>(acc, v, op); break;
	case MPI_UNSIGNED: reduce_into<unsigned>(acc, v, op); break;
	case MPI_INT64_T: case MPI_LONG_LONG: reduce_into<long long>(acc, v, op); break;
	case MPI_UINT64_T: reduce_into<unsigned long long>(acc, v, op); break;
	default:
		std::fprintf(stderr, "tmpi: unsupported reduction type %d\n", t);
		std::abort();
	}
}

}  // namespace

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }

int MPI_Init_thread(int *, char ***, int required, int *provided)
{
	if (provided) *provided = required < MPI_THREAD_SERIALIZED ? required : MPI_THREAD_SERIALIZED;
	return MPI_SUCCESS;
}

int MPI_Finalize(void) { return MPI_Barrier(MPI_COMM_WORLD); }

int MPI_Abort(MPI_Comm, int code)
{
	std::fprintf(stderr, "tmpi: MPI_Abort(%d) from rank %d\n", code, t_rank);
	std::fflush(stderr);
	std::_Exit(code ? code : 1);
}

double MPI_Wtime(void)
{
	using namespace std::chrono;
	return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int MPI_Get_processor_name(char *name, int *len)
{
	gethostname(name, MPI_MAX_PROCESSOR_NAME - 1);
	name[MPI_MAX_PROCESSOR_NAME - 1] = 0;
	if (len) *len = static_cast<int>(std::strlen(name));
	return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
	*rank = my_comm_rank(comm);
	return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
	*size = comm_size(comm);
	return MPI_SUCCESS;
}

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
	const long seq = next_seq(comm);
	const int me = my_comm_rank(comm);
	const int size = comm_size(comm);
	std::unique_lock<std::mutex> lk(g_mu);
	Slot &s = g_slots[{comm, seq}];
	if (s.split.empty()) {
		s.split.assign(size, {0, 0});
		s.newcomm.assign(size, MPI_COMM_NULL);
		s.readers_left = size;
	}
	s.split[me] = {color, key};
	if (++s.arrived == size) {
		// one new communicator per colour, members ordered by (key, rank)
		std::map<int, std::vector<std::tuple<int, int>>> by_color;
		for (int r = 0; r < size; ++r) by_color[s.split[r].first].emplace_back(s.split[r].second, r);
		for (auto &kv : by_color) {
			std::sort(kv.second.begin(), kv.second.end());
			Comm c;
			for (auto &kr : kv.second) c.members.push_back(g_comms.at(comm).members.at(std::get<1>(kr)));
			const int id = static_cast<int>(g_comms.size());
			g_comms.push_back(c);
			for (auto &kr : kv.second) s.newcomm[std::get<1>(kr)] = id;
		}
		s.ready = true;
		g_cv.notify_all();
	}
	g_cv.wait(lk, [&] { return g_slots[{comm, seq}].ready; });
	Slot &t = g_slots[{comm, seq}];
	*newcomm = t.newcomm[me];
	if (--t.readers_left == 0) g_slots.erase({comm, seq});
	return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm)
{
	*comm = MPI_COMM_NULL;
	return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
	if (dest != MPI_PROC_NULL) deliver(comm, dest, tag, buf, static_cast<size_t>(count) * type_size(type));
	*req = new tmpi_request;
	(*req)->done = true;
	return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
	if (dest != MPI_PROC_NULL) deliver(comm, dest, tag, buf, static_cast<size_t>(count) * type_size(type));
	return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req)
{
	tmpi_request *r = new tmpi_request;
	*req = r;
	if (source == MPI_PROC_NULL) {
		r->done = true;
		return MPI_SUCCESS;
	}
	r->kind = tmpi_request::RECV;
	r->buf = buf;
	r->bytes = static_cast<size_t>(count) * type_size(type);
	r->comm = comm;
	r->src = source;
	r->tag = tag;
	Mailbox &box = *g_box.at(t_rank);
	std::lock_guard<std::mutex> lk(box.mu);
	for (auto it = box.unexpected.begin(); it != box.unexpected.end(); ++it) {
		if (it->comm == comm && it->src == source && it->tag == tag) {
			fill_recv(r, *it);
			box.unexpected.erase(it);
			return MPI_SUCCESS;
		}
	}
	box.posted.push_back(r);
	return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status *status)
{
	MPI_Request r;
	MPI_Irecv(buf, count, type, source, tag, comm, &r);
	return MPI_Wait(&r, status);
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void *recvbuf,
	int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status *status)
{
	MPI_Request r;
	MPI_Irecv(recvbuf, recvcount, recvtype, source, recvtag, comm, &r);
	MPI_Send(sendbuf, sendcount, sendtype, dest, sendtag, comm);
	return MPI_Wait(&r, status);
}

int MPI_Wait(MPI_Request *req, MPI_Status *status)
{
	if (*req) {
		wait_one(*req);
		delete *req;
		*req = MPI_REQUEST_NULL;
	}
	set_status(status);
	return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
	for (int i = 0; i < count; ++i) MPI_Wait(&reqs[i], statuses ? &statuses[i] : MPI_STATUS_IGNORE);
	return MPI_SUCCESS;
}

int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status)
{
	if (!*req || progress(*req)) {
		delete *req;
		*req = MPI_REQUEST_NULL;
		*flag = 1;
		set_status(status);
	} else {
		*flag = 0;
	}
	return MPI_SUCCESS;
}

int MPI_Testall(int count, MPI_Request *reqs, int *flag, MPI_Status *statuses)
{
	bool all = true;
	for (int i = 0; i < count; ++i)
		if (!progress(reqs[i])) all = false;
	if (all) {
		for (int i = 0; i < count; ++i) {
			delete reqs[i];
			reqs[i] = MPI_REQUEST_NULL;
			if (statuses) set_status(&statuses[i]);
		}
	}
	*flag = all ? 1 : 0;
	return MPI_SUCCESS;
}

int MPI_Ibcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request *req)
{
	const long seq = next_seq(comm);
	const int me = my_comm_rank(comm);
	const int size = comm_size(comm);
	const size_t bytes = static_cast<size_t>(count) * type_size(type);
	tmpi_request *r = new tmpi_request;
	*req = r;
	if (size == 1 || me == root) {
		if (size > 1) {
			std::lock_guard<std::mutex> lk(g_mu);
			Slot &s = g_slots[{comm, seq}];
			s.data.assign(static_cast<const char *>(buf), static_cast<const char *>(buf) + bytes);
			s.readers_left = size - 1;
			s.ready = true;
			g_cv.notify_all();
		}
		r->done = true;
		return MPI_SUCCESS;
	}
	r->kind = tmpi_request::BCAST;
	r->buf = buf;
	r->bytes = bytes;
	r->comm = comm;
	r->seq = seq;
	r->root = root;
	return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
	MPI_Request r;
	MPI_Ibcast(buf, count, type, root, comm, &r);
	return MPI_Wait(&r, MPI_STATUS_IGNORE);
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
	const long seq = next_seq(comm);
	const int me = my_comm_rank(comm);
	const int size = comm_size(comm);
	const size_t bytes = static_cast<size_t>(count) * type_size(type);
	const char *src = static_cast<const char *>(sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf);
	std::unique_lock<std::mutex> lk(g_mu);
	Slot &s = g_slots[{comm, seq}];
	if (s.contrib.empty()) {
		s.contrib.resize(size);
		s.readers_left = size;
	}
	s.contrib[me].assign(src, src + bytes);
	if (++s.arrived == size) {
		// contributions folded in rank order: deterministic
		s.data = s.contrib[0];
		for (int r = 1; r < size; ++r) reduce_typed(s.data, s.contrib[r], type, op);
		s.ready = true;
		g_cv.notify_all();
	}
	g_cv.wait(lk, [&] { return g_slots[{comm, seq}].ready; });
	Slot &t = g_slots[{comm, seq}];
	if (bytes) std::memcpy(recvbuf, t.data.data(), bytes);
	if (--t.readers_left == 0) g_slots.erase({comm, seq});
	return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm)
{
	int z = 0, o = 0;
	return MPI_Allreduce(&z, &o, 1, MPI_INT, MPI_SUM, comm);
}

// The solution vector from ref_xdump.cpp: each rank stores the entries it
// owns; the last rank to finish writes the file named by TMPI_XDUMP.
void tmpi_xdump_put(long long first, const double *x, int count, long long n)
{
	std::lock_guard<std::mutex> lk(g_x_mu);
	if (static_cast<long long>(g_x.size()) != n) g_x.assign(static_cast<size_t>(n), 0.0);
	std::memcpy(g_x.data() + first, x, sizeof(double) * static_cast<size_t>(count));
}

void tmpi_xdump_rank_done(void)
{
	std::lock_guard<std::mutex> lk(g_x_mu);
	if (++g_x_done < g_world) return;
	const char *path = std::getenv("TMPI_XDUMP");
	if (!path || !*path) return;
	FILE *f = std::fopen(path, "wb");
	if (!f) return;
	std::fwrite(g_x.data(), sizeof(double), g_x.size(), f);
	std::fclose(f);
}

// The factored matrix from ref_xdump.cpp (TMPI_LUDUMP), gathered the same way.
void tmpi_ludump_put(long long row0, long long col0, const float *blk, long long ld, int b, long long n)
{
	if (!std::getenv("TMPI_LUDUMP")) return;
	std::lock_guard<std::mutex> lk(g_x_mu);
	if (static_cast<long long>(g_lu.size()) != n * n) g_lu.assign(static_cast<size_t>(n * n), 0.f);
	for (int jj = 0; jj < b; ++jj)
		std::memcpy(g_lu.data() + (col0 + jj) * n + row0, blk + jj * ld, sizeof(float) * static_cast<size_t>(b));
}

void tmpi_ludump_rank_done(void)
{
	std::lock_guard<std::mutex> lk(g_x_mu);
	if (++g_lu_done < g_world) return;
	const char *path = std::getenv("TMPI_LUDUMP");
	if (!path || !*path) return;
	FILE *f = std::fopen(path, "wb");
	if (!f) return;
	std::fwrite(g_lu.data(), sizeof(float), g_lu.size(), f);
	std::fclose(f);
}

}  // extern "C"

int main(int argc, char **argv)
{
	const char *np = std::getenv("TMPI_NP");
	g_world = np ? std::atoi(np) : 4;
	if (g_world < 1) g_world = 1;
	Comm world;
	for (int r = 0; r < g_world; ++r) {
		world.members.push_back(r);
		g_box.emplace_back(new Mailbox);
	}
	g_comms.push_back(world);
	std::vector<int> rc(g_world, 0);
	std::vector<std::thread> ranks;
	for (int r = 0; r < g_world; ++r)
		ranks.emplace_back([&, r] {
			t_rank = r;
			rc[r] = hplai_rank_main(argc, argv);
		});
	for (auto &t : ranks) t.join();
	return rc[0];
}
