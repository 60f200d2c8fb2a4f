// shard.cpp — see shard.h.
#include "shard.h"

#include <arpa/inet.h>
#include <netdb.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <unistd.h>

#include <cerrno>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace fps {

namespace {

const uint32_t kMagic = 0x46505353u;   // "FPSS"

int envInt(const char* a, const char* b, int dflt)
{
    const char* v = std::getenv(a);
    if (!v && b) v = std::getenv(b);
    return v ? std::atoi(v) : dflt;
}

using Clock = std::chrono::steady_clock;

double secondsLeft(Clock::time_point deadline)
{
    return std::chrono::duration<double>(deadline - Clock::now()).count();
}

// Waits until fd is readable (events = POLLIN) or writable (POLLOUT) or the deadline passes.
bool waitFd(int fd, short events, Clock::time_point deadline)
{
    for (;;) {
        const double left = secondsLeft(deadline);
        if (left <= 0) return false;
        pollfd p = {fd, events, 0};
        const int r = ::poll(&p, 1, (int)std::min(left * 1000.0 + 1, 1000.0));
        if (r > 0) return true;
        if (r < 0 && errno != EINTR) return false;
    }
}

bool sendAll(int fd, const void* buf, size_t n, Clock::time_point deadline)
{
    const char* p = static_cast<const char*>(buf);
    while (n > 0) {
        if (!waitFd(fd, POLLOUT, deadline)) return false;
        const ssize_t k = ::send(fd, p, n, MSG_NOSIGNAL);
        if (k < 0) {
            if (errno == EINTR || errno == EAGAIN) continue;
            return false;
        }
        p += k;
        n -= (size_t)k;
    }
    return true;
}

bool recvAll(int fd, void* buf, size_t n, Clock::time_point deadline)
{
    char* p = static_cast<char*>(buf);
    while (n > 0) {
        if (!waitFd(fd, POLLIN, deadline)) return false;
        const ssize_t k = ::recv(fd, p, n, 0);
        if (k == 0) return false;                      // peer closed
        if (k < 0) {
            if (errno == EINTR || errno == EAGAIN) continue;
            return false;
        }
        p += k;
        n -= (size_t)k;
    }
    return true;
}

struct Header {
    uint32_t magic;
    int32_t rank;
    int64_t count;
};

bool resolve(const std::string& addr, int port, sockaddr_in& sa)
{
    std::memset(&sa, 0, sizeof sa);
    sa.sin_family = AF_INET;
    sa.sin_port = htons((uint16_t)port);
    if (inet_pton(AF_INET, addr.c_str(), &sa.sin_addr) == 1) return true;
    addrinfo hints = {}, *res = nullptr;
    hints.ai_family = AF_INET;
    if (getaddrinfo(addr.c_str(), nullptr, &hints, &res) != 0 || !res) return false;
    sa.sin_addr = reinterpret_cast<sockaddr_in*>(res->ai_addr)->sin_addr;
    freeaddrinfo(res);
    return true;
}

}  // namespace

ShardEnv ShardEnv::fromEnvironment()
{
    ShardEnv e;
    e.world = envInt("WORLD_SIZE", "OMPI_COMM_WORLD_SIZE", 1);
    e.rank = envInt("RANK", "OMPI_COMM_WORLD_RANK", 0);
    e.local = envInt("LOCAL_RANK", "OMPI_COMM_WORLD_LOCAL_RANK", e.rank);
    if (const char* a = std::getenv("MASTER_ADDR")) e.addr = a;
    if (const char* p = std::getenv("FPS_SHARD_PORT")) e.port = std::atoi(p);
    else if (const char* m = std::getenv("MASTER_PORT")) e.port = std::atoi(m) + 1;
    if (const char* t = std::getenv("FPS_SHARD_TIMEOUT")) e.timeout_s = std::atof(t);
    return e;
}

void shardRange(long long nTraj, int rank, int world, long long& first, long long& end)
{
    const long long per = nTraj / world, extra = nTraj % world;
    const long long firstBig = world - extra;            // ranks >= firstBig take per + 1
    if (rank < firstBig) {
        first = rank * per;
        end = first + per;
    } else {
        first = firstBig * per + (rank - firstBig) * (per + 1);
        end = first + per + 1;
    }
}

int shardSum(const ShardEnv& env, std::vector<double>& data, std::string& err)
{
    if (env.world <= 1) return 0;
    if (env.rank < 0 || env.rank >= env.world) { err = "rank outside [0, world)"; return -1; }
    const auto deadline = Clock::now() + std::chrono::milliseconds((long long)(env.timeout_s * 1000.0));
    const int64_t count = (int64_t)data.size();
    sockaddr_in sa;
    if (!resolve(env.addr, env.port, sa)) { err = "cannot resolve " + env.addr; return -1; }

    if (env.rank == 0) {
        const int ls = ::socket(AF_INET, SOCK_STREAM, 0);
        if (ls < 0) { err = "socket: " + std::string(std::strerror(errno)); return -1; }
        int one = 1;
        setsockopt(ls, SOL_SOCKET, SO_REUSEADDR, &one, sizeof one);
        if (::bind(ls, reinterpret_cast<sockaddr*>(&sa), sizeof sa) != 0 || ::listen(ls, env.world) != 0) {
            err = "cannot listen on " + env.addr + ":" + std::to_string(env.port) + ": " + std::strerror(errno);
            ::close(ls);
            return -1;
        }
        std::vector<int> peer(env.world, -1);
        std::vector<std::vector<double>> bufs(env.world);
        int rc = 0;
        for (int got = 1; got < env.world && rc == 0; ++got) {
            if (!waitFd(ls, POLLIN, deadline)) { err = "timed out waiting for the other ranks"; rc = -2; break; }
            const int fd = ::accept(ls, nullptr, nullptr);
            if (fd < 0) { err = "accept: " + std::string(std::strerror(errno)); rc = -1; break; }
            Header h;
            if (!recvAll(fd, &h, sizeof h, deadline) || h.magic != kMagic || h.rank <= 0 || h.rank >= env.world ||
                peer[h.rank] >= 0 || h.count != count) {
                err = "bad shard message (rank, size or protocol mismatch)";
                ::close(fd);
                rc = -1;
                break;
            }
            peer[h.rank] = fd;
            bufs[h.rank].resize((size_t)count);
            if (!recvAll(fd, bufs[h.rank].data(), sizeof(double) * (size_t)count, deadline)) {
                err = "timed out receiving rank " + std::to_string(h.rank);
                rc = -2;
            }
        }
        if (rc == 0) {
            for (int r = 1; r < env.world; ++r)          // rank order: 0 (own data), 1, 2, ...
                for (int64_t q = 0; q < count; ++q) data[(size_t)q] += bufs[r][(size_t)q];
            for (int r = 1; r < env.world && rc == 0; ++r)
                if (!sendAll(peer[r], data.data(), sizeof(double) * (size_t)count, deadline)) {
                    err = "timed out sending the sum to rank " + std::to_string(r);
                    rc = -2;
                }
        }
        for (int fd : peer)
            if (fd >= 0) ::close(fd);
        ::close(ls);
        return rc;
    }

    // other ranks: connect (rank 0 may not listen yet), send, receive the sum
    int fd = -1;
    while (fd < 0) {
        if (secondsLeft(deadline) <= 0) { err = "timed out connecting to rank 0 at " + env.addr; return -2; }
        fd = ::socket(AF_INET, SOCK_STREAM, 0);
        if (fd < 0) { err = "socket: " + std::string(std::strerror(errno)); return -1; }
        if (::connect(fd, reinterpret_cast<sockaddr*>(&sa), sizeof sa) != 0) {
            ::close(fd);
            fd = -1;
            std::this_thread::sleep_for(std::chrono::milliseconds(50));
        }
    }
    int one = 1;
    setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
    const Header h = {kMagic, (int32_t)env.rank, count};
    int rc = 0;
    if (!sendAll(fd, &h, sizeof h, deadline) || !sendAll(fd, data.data(), sizeof(double) * (size_t)count, deadline)) {
        err = "lost the connection to rank 0 while sending";
        rc = -2;
    } else if (!recvAll(fd, data.data(), sizeof(double) * (size_t)count, deadline)) {
        err = "no sum from rank 0 before the deadline";
        rc = -2;
    }
    ::close(fd);
    return rc;
}

}  // namespace fps
