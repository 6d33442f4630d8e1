// cuopus_decode: the command-line tool and unix-socket daemon of libcuopus.
//
// Same modes, flags, files and protocol as the reference's decode_cli.cu
// (:3-33, :680-734), built on the library's C ABI:
//
//   cuopus_decode <packets.blob> <chains.bin> <out.pcm> [stride]
//       legacy blob mode: a 'CUOP' packet blob (u32 magic, u32 n, u32 len[n],
//       bytes) and a 'CUC2' chain table (u32 magic, u32 n, {first, npkts,
//       trim, keep}[n]) -> int16 PCM of every chain's keep window, in order
//   cuopus_decode --ogg <in.ogg> [out|-] [--seg S] [--preroll MS] [--stride N]
//                 [--f16k] [--dump-blob F] [--dump-chains F]
//       demux + decode an Ogg Opus file: int16 48 kHz playable PCM, or with
//       --f16k float32 16 kHz (on-device resample, (play48 - 48) / 3 samples);
//       "-" or no output = demux only; the dumps write the blob / CUC2 table
//   cuopus_decode --serve <unix_socket>
//       daemon, one request line per connection:
//         PING                                          -> PONG 2
//         DECODE <seg_s> <preroll_ms> <stride> <ogg> <out.pcm>
//         DECODE16F <seg_s> <preroll_ms> <stride> <ogg> <out.f32>
//             -> OK <samples> <play48> <kernel_ms> <wall_ms> <demux_ms>
//                   <h2d_ms> <d2h_ms> <resample_ms> <fwrite_ms>
//             -> ERR <message>                (the daemon keeps serving)
//         QUIT                                          -> BYE, exit 0
//       idle exit after CUOPUS_SERVE_IDLE_S seconds (default 600).
//
// Differences, all extensions: stereo streams decode in the int16 modes
// (interleaved), and the daemon keeps serving after a CUDA error is reported
// (ERR, the context state is reported by the next request).
// Exit codes: 0 ok, 1 decode / stream failure, 2 usage or I/O error.
#include <cuda_runtime.h>
#include <errno.h>
#include <poll.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/socket.h>
#include <sys/time.h>
#include <sys/un.h>
#include <time.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "cuopus.h"

namespace {

const int DEF_STRIDE = 32;
const double DEF_PREROLL_MS = 250.0;

double now_ms()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

bool read_file(const char *path, std::vector<uint8_t> &out, std::string &err)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        err = std::string("cannot open ") + path + ": " + strerror(errno);
        return false;
    }
    out.clear();
    uint8_t buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, f)) > 0) out.insert(out.end(), buf, buf + r);
    bool ok = !ferror(f);
    fclose(f);
    if (!ok) err = std::string("read error on ") + path;
    return ok;
}

bool write_file(const char *path, const void *p, size_t bytes, std::string &err)
{
    FILE *f = fopen(path, "wb");
    if (!f) {
        err = std::string("cannot create ") + path + ": " + strerror(errno);
        return false;
    }
    bool ok = fwrite(p, 1, bytes, f) == bytes;
    ok = (fclose(f) == 0) && ok;
    if (!ok) err = std::string("write error on ") + path;
    return ok;
}

void set_env_params(double seg_s, double preroll_ms, unsigned stride)
{
    char v[64];
    snprintf(v, sizeof v, "%.9g", seg_s);
    setenv("CUOPUS_SEG_S", v, 1);
    snprintf(v, sizeof v, "%.9g", preroll_ms);
    setenv("CUOPUS_PREROLL_MS", v, 1);
    snprintf(v, sizeof v, "%u", stride);
    setenv("CUOPUS_STRIDE", v, 1);
}

struct Report {
    unsigned long long out_samples = 0;
    long long play48 = 0;
    cuopus_stats st{};
    double d2h_ms = 0, fwrite_ms = 0, wall_ms = 0;
};

// Decode an in-memory Ogg stream to `out` (int16 48 kHz or float32 16 kHz).
// Returns 0, 1 (stream / decode failure) or 2 (I/O).
int decode_ogg(const std::vector<uint8_t> &ogg, const char *out, bool f16k, Report &rep, std::string &err)
{
    char eb[512];
    double t0 = now_ms();
    const uint8_t *op = ogg.data();
    size_t on = ogg.size();
    int rc;
    std::vector<uint8_t> host;
    size_t bytes = 0;
    if (f16k) {
        int64_t n16 = 0;
        if ((rc = cuopus_probe(op, on, &n16, eb, sizeof eb))) {
            err = eb;
            return 1;
        }
        float *dev = nullptr;
        if (n16 > 0 && cudaMalloc(&dev, (size_t)n16 * 4) != cudaSuccess) {
            err = "cudaMalloc failed";
            return 1;
        }
        int64_t len = 0;
        rc = cuopus_decode_f16k_on(op, on, dev, (size_t)n16, &len, nullptr, eb, sizeof eb);
        if (rc) {
            err = eb;
            cudaFree(dev);
            return 1;
        }
        cuopus_last_stats(&rep.st);
        double t1 = now_ms();
        host.resize((size_t)len * 4);
        if (len && cudaMemcpy(host.data(), dev, (size_t)len * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            err = "device to host copy failed";
            cudaFree(dev);
            return 1;
        }
        rep.d2h_ms = now_ms() - t1;
        cudaFree(dev);
        bytes = host.size();
        rep.out_samples = (unsigned long long)len;
    } else {
        int64_t play = 0;
        int32_t ch = 0;
        if ((rc = cuopus_probe_pcm(op, on, &play, &ch, eb, sizeof eb))) {
            err = eb;
            return 1;
        }
        size_t elems = (size_t)play * (size_t)ch;
        int16_t *dev = nullptr;
        if (elems && cudaMalloc(&dev, elems * 2) != cudaSuccess) {
            err = "cudaMalloc failed";
            return 1;
        }
        const uint8_t *oggs[1] = {op};
        size_t ns[1] = {on};
        int16_t *outs[1] = {dev};
        size_t caps[1] = {elems};
        int64_t lens[1] = {0};
        int32_t chs[1] = {0};
        rc = cuopus_decode_i16_multi(oggs, ns, 1, outs, caps, lens, chs, nullptr, eb, sizeof eb);
        if (rc) {
            err = eb;
            cudaFree(dev);
            return 1;
        }
        cuopus_last_stats(&rep.st);
        double t1 = now_ms();
        host.resize(elems * 2);
        if (elems && cudaMemcpy(host.data(), dev, elems * 2, cudaMemcpyDeviceToHost) != cudaSuccess) {
            err = "device to host copy failed";
            cudaFree(dev);
            return 1;
        }
        rep.d2h_ms = now_ms() - t1;
        cudaFree(dev);
        bytes = host.size();
        rep.out_samples = (unsigned long long)lens[0] * (unsigned long long)chs[0];
    }
    double t2 = now_ms();
    if (!write_file(out, host.data(), bytes, err)) return 2;
    rep.fwrite_ms = now_ms() - t2;
    rep.play48 = rep.st.play48;
    rep.wall_ms = now_ms() - t0;
    return 0;
}

int run_ogg_once(const char *ogg_path, const char *out, double seg_s, double preroll_ms, unsigned stride,
                 bool f16k, const char *dump_blob, const char *dump_chains)
{
    std::string err;
    std::vector<uint8_t> ogg;
    if (!read_file(ogg_path, ogg, err)) {
        fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
        return 2;
    }
    set_env_params(seg_s, preroll_ms, stride);
    double t0 = now_ms();
    char eb[512];
    int64_t npk = 0, nch = 0, nb = 0, play = 0;
    int32_t ch = 0;
    int rc = cuopus_index(ogg.data(), ogg.size(), seg_s, preroll_ms, 0, &npk, &nch, &nb, &ch, &play, nullptr,
                          nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, eb, sizeof eb);
    if (rc) {
        fprintf(stderr, "cuopus_decode: demux: %s\n", eb);
        return 1;
    }
    double t_demux = now_ms() - t0;
    if (dump_blob || dump_chains) {
        std::vector<uint8_t> blob((size_t)nb + 1);
        std::vector<uint64_t> off((size_t)npk + 1);
        std::vector<uint32_t> len((size_t)npk + 1), first((size_t)nch + 1), npkts((size_t)nch + 1),
            trim((size_t)nch + 1), keep((size_t)nch + 1);
        rc = cuopus_index(ogg.data(), ogg.size(), seg_s, preroll_ms, 0, &npk, &nch, &nb, &ch, &play, blob.data(),
                          off.data(), len.data(), first.data(), npkts.data(), trim.data(), keep.data(), eb,
                          sizeof eb);
        if (rc) {
            fprintf(stderr, "cuopus_decode: demux: %s\n", eb);
            return 1;
        }
        if (dump_blob) {
            std::vector<uint8_t> f;
            uint32_t hdr[2] = {0x504F5543u /* "CUOP" */, (uint32_t)npk};
            f.insert(f.end(), (uint8_t *)hdr, (uint8_t *)(hdr + 2));
            f.insert(f.end(), (uint8_t *)len.data(), (uint8_t *)(len.data() + npk));
            f.insert(f.end(), blob.data(), blob.data() + nb);
            if (!write_file(dump_blob, f.data(), f.size(), err)) {
                fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
                return 1;
            }
        }
        if (dump_chains) {
            std::vector<uint32_t> f = {0x32435543u /* "CUC2" */, (uint32_t)nch};
            for (int64_t i = 0; i < nch; i++) {
                f.push_back(first[i]);
                f.push_back(npkts[i]);
                f.push_back(trim[i]);
                f.push_back(keep[i]);
            }
            if (!write_file(dump_chains, f.data(), f.size() * 4, err)) {
                fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
                return 1;
            }
        }
    }
    if (!out || !strcmp(out, "-")) {
        printf("cuopus_decode: demux %s: %lld packets, %lld chains, %lld playable samples, %.1f ms\n", ogg_path,
               (long long)npk, (long long)nch, (long long)play, t_demux);
        return 0;
    }
    if (f16k && ch != 1) {
        fprintf(stderr, "cuopus_decode: only mono supported with --f16k (channels=%d)\n", ch);
        return 1;
    }
    Report rep;
    rc = decode_ogg(ogg, out, f16k, rep, err);
    if (rc) {
        fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
        return rc;
    }
    printf("cuopus_decode: %lld chains (stride %u), %lld packets, %llu samples out (%s)\n",
           (long long)rep.st.chains, stride, (long long)rep.st.packets, rep.out_samples,
           f16k ? "float32 @16k" : "int16 @48k");
    printf("cuopus_decode: demux %.1f ms, h2d %.1f, kernel %.1f, resample %.1f, d2h %.1f, fwrite %.1f, wall %.1f ms\n",
           rep.st.demux_ms, rep.st.h2d_ms, rep.st.kernel_ms, rep.st.resample_ms, rep.d2h_ms, rep.fwrite_ms,
           rep.wall_ms + t_demux);
    return 0;
}

// ------------------------------------------------------------------ legacy blob mode

template <class T> bool take(const std::vector<uint8_t> &b, size_t &o, T &v)
{
    if (o + sizeof(T) > b.size()) return false;
    memcpy(&v, b.data() + o, sizeof(T));
    o += sizeof(T);
    return true;
}

int run_blob(const char *blob_path, const char *chains_path, const char *out, unsigned stride)
{
    std::string err;
    std::vector<uint8_t> bf, cf;
    if (!read_file(blob_path, bf, err) || !read_file(chains_path, cf, err)) {
        fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
        return 2;
    }
    size_t o = 0;
    uint32_t magic = 0, n = 0;
    if (!take(bf, o, magic) || magic != 0x504F5543u || !take(bf, o, n)) {
        fprintf(stderr, "cuopus_decode: %s: bad magic (want CUOP)\n", blob_path);
        return 2;
    }
    std::vector<uint32_t> len(n);
    std::vector<uint64_t> off(n);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (!take(bf, o, len[i])) {
            fprintf(stderr, "cuopus_decode: %s: truncated\n", blob_path);
            return 2;
        }
        off[i] = total;
        total += len[i];
    }
    if (o + total > bf.size()) {
        fprintf(stderr, "cuopus_decode: %s: truncated\n", blob_path);
        return 2;
    }
    const uint8_t *data = bf.data() + o;
    size_t co = 0;
    uint32_t nch = 0;
    if (!take(cf, co, magic) || magic != 0x32435543u || !take(cf, co, nch)) {
        fprintf(stderr, "cuopus_decode: %s: bad magic (want CUC2)\n", chains_path);
        return 2;
    }
    std::vector<uint32_t> first(nch), npk(nch);
    std::vector<uint64_t> trim(nch), keep(nch), out_off(nch);
    std::vector<uint8_t> chans(nch, 1);
    uint64_t elems = 0;
    for (uint32_t i = 0; i < nch; i++) {
        uint32_t t = 0, k = 0;
        if (!take(cf, co, first[i]) || !take(cf, co, npk[i]) || !take(cf, co, t) || !take(cf, co, k)) {
            fprintf(stderr, "cuopus_decode: %s: truncated\n", chains_path);
            return 2;
        }
        if ((uint64_t)first[i] + npk[i] > n) {
            fprintf(stderr, "cuopus_decode: chain %u outside the blob\n", i);
            return 2;
        }
        trim[i] = t;
        keep[i] = k;
        out_off[i] = elems;
        elems += k;
    }
    double t0 = now_ms();
    // device copies of the tables
    void *d[9] = {};
    size_t sz[9] = {total + 16, 8ull * n + 8, 4ull * n + 4, 4ull * nch + 4, 4ull * nch + 4, nch + 1ull,
                    8ull * nch + 8, 8ull * nch + 8, 8ull * nch + 8};
    const void *src[9] = {data, off.data(), len.data(), first.data(), npk.data(), chans.data(), trim.data(),
                          keep.data(), out_off.data()};
    size_t cp[9] = {total, 8ull * n, 4ull * n, 4ull * nch, 4ull * nch, nch, 8ull * nch, 8ull * nch, 8ull * nch};
    int16_t *pcm = nullptr;
    uint32_t *res = nullptr;
    int rc = 0;
    for (int i = 0; i < 9 && !rc; i++) {
        if (cudaMalloc(&d[i], sz[i]) != cudaSuccess ||
            (cp[i] && cudaMemcpy(d[i], src[i], cp[i], cudaMemcpyHostToDevice) != cudaSuccess))
            rc = 1;
    }
    if (!rc && (cudaMalloc(&pcm, 2 * elems + 16) != cudaSuccess || cudaMalloc(&res, 16ull * nch + 16) != cudaSuccess))
        rc = 1;
    std::vector<int16_t> host(elems);
    float kms = 0;
    if (!rc) {
        cuopus_batch b;
        memset(&b, 0, sizeof b);
        b.data = (const uint8_t *)d[0];
        b.off = (const uint64_t *)d[1];
        b.len = (const uint32_t *)d[2];
        b.first = (const uint32_t *)d[3];
        b.npkts = (const uint32_t *)d[4];
        b.channels = (const uint8_t *)d[5];
        b.trim = (const uint64_t *)d[6];
        b.keep = (const uint64_t *)d[7];
        b.out_off = (const uint64_t *)d[8];
        b.out = pcm;
        b.res = res;
        b.nchains = (int32_t)nch;
        int w = 1;
        while (w * 2 <= (int)stride && w < 32) w *= 2;
        b.width = w;
        b.schedule = 1;
        char eb[512];
        if (cuopus_decode_batch(&b, nullptr, &kms, eb, sizeof eb)) {
            fprintf(stderr, "cuopus_decode: %s\n", eb);
            rc = 1;
        }
    }
    if (!rc) {
        std::vector<uint32_t> r(4ull * nch);
        if (cudaMemcpy(r.data(), res, 16ull * nch, cudaMemcpyDeviceToHost) != cudaSuccess ||
            (elems && cudaMemcpy(host.data(), pcm, 2 * elems, cudaMemcpyDeviceToHost) != cudaSuccess))
            rc = 1;
        for (uint32_t i = 0; i < nch && !rc; i++) {
            uint64_t cap = 0;
            for (uint32_t k = 0; k < npk[i]; k++) {
                const uint8_t *p = data + off[first[i] + k];
                uint32_t L = len[first[i] + k];
                if (!L) continue;
                static const int qms[32] = {40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 40, 80,
                                            10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80};
                int code = p[0] & 3;
                int nf = code == 0 ? 1 : code < 3 ? 2 : (L > 1 ? (p[1] & 0x3F) : 0);
                cap += (uint64_t)qms[p[0] >> 3] * 12 * nf;
            }
            if ((int32_t)r[4 * i] != 0 || r[4 * i + 1] != cap) {
                fprintf(stderr, "cuopus_decode: chain %u failed (status %d, %u of %llu samples)\n", i,
                        (int32_t)r[4 * i], r[4 * i + 1], (unsigned long long)cap);
                rc = 1;
            }
        }
    }
    for (void *p : d) cudaFree(p);
    cudaFree(pcm);
    cudaFree(res);
    if (rc) return rc;
    if (!write_file(out, host.data(), 2 * elems, err)) {
        fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
        return 2;
    }
    printf("cuopus_decode: %u chains (stride %u), %u packets, %llu samples out (%.3f s @48k)\n", nch, stride, n,
           (unsigned long long)elems, elems / 48000.0);
    printf("cuopus_decode: kernel %.1f ms, wall %.1f ms\n", kms, now_ms() - t0);
    return 0;
}

// ------------------------------------------------------------------ daemon
//
// The daemon is an event loop over the listening socket and every open client
// connection at once (poll), with the decoding handed to the library's
// continuous-batching server (cuopus_server_*).  A connection's request line
// is parsed into a Request; a DECODE request's file is read, probed and
// submitted, and the connection is answered when the server completes it, so
// requests from several clients are admitted together and decode in the same
// waves on the GPU.  One server is kept per distinct (output format, chain
// length, preroll, lanes per chain), created on first use and kept resident,
// each with a device arena of CUOPUS_SERVE_BUDGET_MB (default 4096).
//
// Reply fields of OK, in order: int16 values (or float32 samples) written,
// playable samples per channel at 48 kHz, decode ms (submit to completion in
// the server: queueing, host->device copy, decode and resample), request wall
// ms (line received to reply), file read + demux + submit ms, host->device
// ms and resample ms (both 0.0: they are inside the decode ms), result copy
// ms, file write ms.
//
// A connection that has not sent a complete line 30 s after it was accepted
// is closed.  QUIT is answered at once; requests already submitted still
// complete and are answered, then the daemon exits 0.  With no connection
// open and nothing in flight for CUOPUS_SERVE_IDLE_S seconds (default 600) it
// exits 0 as well.

enum class Verb { None, Ping, Quit, Decode, Malformed, Unknown };

struct Request {
    Verb verb = Verb::None;
    bool f16k = false;
    double seg_s = 0, preroll_ms = 0;
    unsigned stride = DEF_STRIDE;
    std::string in, out;
};

// One request line -> Request.  Fields are separated by blanks; paths may not
// contain blanks (the protocol's own limit).
Request parse_request(const std::string &line)
{
    std::vector<std::string> tok;
    size_t i = 0;
    auto blank = [](char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; };
    while (i < line.size()) {
        while (i < line.size() && blank(line[i])) i++;
        size_t j = i;
        while (j < line.size() && !blank(line[j])) j++;
        if (j > i) tok.push_back(line.substr(i, j - i));
        i = j;
    }
    Request r;
    if (tok.empty()) return r;
    r.verb = Verb::Unknown;
    if (tok[0] == "PING") {
        r.verb = Verb::Ping;
    } else if (tok[0] == "QUIT") {
        r.verb = Verb::Quit;
    } else if (tok[0] == "DECODE" || tok[0] == "DECODE16F") {
        r.f16k = tok[0] == "DECODE16F";
        r.verb = Verb::Malformed;
        if (tok.size() != 6) return r;
        char *end = nullptr;
        r.seg_s = strtod(tok[1].c_str(), &end);
        if (*end || !(r.seg_s > 0)) return r;
        r.preroll_ms = strtod(tok[2].c_str(), &end);
        if (*end || r.preroll_ms < 0) return r;
        long st = strtol(tok[3].c_str(), &end, 10);
        if (*end || st < 0) return r;
        r.stride = (unsigned)(st < 1 ? 1 : st);
        r.in = tok[4];
        r.out = tok[5];
        r.verb = Verb::Decode;
    }
    return r;
}

int width_of(unsigned stride)
{
    int w = 1;
    while (w * 2 <= (int)stride && w < 32) w *= 2;
    return w;
}

// Resident decode servers, one per request configuration.
class ServerPool {
  public:
    ServerPool() = default;
    ServerPool(const ServerPool &) = delete;
    ServerPool &operator=(const ServerPool &) = delete;
    ~ServerPool()
    {
        for (auto &e : servers_) cuopus_server_destroy(e.srv);
    }

    cuopus_server *get(const Request &r, std::string &err)
    {
        const int w = width_of(r.stride);
        for (auto &e : servers_)
            if (e.f16k == r.f16k && e.seg == r.seg_s && e.pre == r.preroll_ms && e.width == w) return e.srv;
        cuopus_server_config cfg;
        memset(&cfg, 0, sizeof cfg);
        long long mb = 4096;
        if (const char *v = getenv("CUOPUS_SERVE_BUDGET_MB"))
            if (atoll(v) > 0) mb = atoll(v);
        cfg.budget_bytes = (int64_t)mb << 20;
        cfg.width = w;
        cfg.seg_s = r.seg_s;
        cfg.preroll_ms = r.preroll_ms;
        cfg.f16k = r.f16k ? 1 : 0;
        cuopus_server *s = nullptr;
        char eb[512];
        if (cuopus_server_create(&cfg, &s, eb, sizeof eb)) {
            err = eb;
            return nullptr;
        }
        servers_.push_back({r.f16k, r.seg_s, r.preroll_ms, w, s});
        return s;
    }

  private:
    struct Entry {
        bool f16k;
        double seg, pre;
        int width;
        cuopus_server *srv;
    };
    std::vector<Entry> servers_;
};

struct Client {
    int fd = -1;
    std::string inbuf;
    double accepted_ms = 0;
    double line_ms = 0;         // request line complete
    bool in_server = false;     // a DECODE is submitted and not yet answered
    cuopus_server *srv = nullptr;
    uint64_t id = 0;
    Request req;
    size_t out_bytes = 0;
    std::vector<uint8_t> host;  // the result, copied out by the server
    long long play48 = 0;
    double prep_ms = 0;
    bool done = false;          // answered: close and drop
};

bool send_all(int fd, const std::string &msg)
{
    size_t o = 0;
    while (o < msg.size()) {
        ssize_t w = send(fd, msg.data() + o, msg.size() - o, MSG_NOSIGNAL);
        if (w < 0 && errno == EINTR) continue;
        if (w <= 0) return false;
        o += (size_t)w;
    }
    return true;
}

class Daemon {
  public:
    Daemon(const char *path, int idle_s) : path_(path), idle_s_(idle_s) {}
    int run();

  private:
    bool listen_on_path();
    void on_readable(Client &c);
    void on_line(Client &c, const std::string &line);
    void submit(Client &c);
    void collect();
    void answer(Client &c, const std::string &text);

    static const size_t kMaxLine = 8192;
    static constexpr double kLineTimeoutMs = 30000.0;
    std::string path_;
    int idle_s_;
    int lfd_ = -1;
    bool quitting_ = false;
    double last_busy_ms_ = 0;
    std::vector<Client> clients_;
    ServerPool pool_;
};

bool Daemon::listen_on_path()
{
    struct sockaddr_un addr;
    memset(&addr, 0, sizeof addr);
    if (path_.size() >= sizeof(addr.sun_path)) {
        fprintf(stderr, "cuopus_decode: socket path longer than %zu bytes\n", sizeof(addr.sun_path) - 1);
        return false;
    }
    addr.sun_family = AF_UNIX;
    memcpy(addr.sun_path, path_.c_str(), path_.size() + 1);
    lfd_ = socket(AF_UNIX, SOCK_STREAM | SOCK_NONBLOCK, 0);
    if (lfd_ < 0) {
        perror("cuopus_decode: socket");
        return false;
    }
    unlink(path_.c_str());
    if (bind(lfd_, (struct sockaddr *)&addr, sizeof addr) != 0 || listen(lfd_, 64) != 0) {
        perror("cuopus_decode: bind / listen");
        close(lfd_);
        lfd_ = -1;
        return false;
    }
    return true;
}

void Daemon::answer(Client &c, const std::string &text)
{
    send_all(c.fd, text);
    c.done = true;
}

void Daemon::on_readable(Client &c)
{
    char buf[4096];
    ssize_t r = recv(c.fd, buf, sizeof buf, MSG_DONTWAIT);
    if (r < 0 && (errno == EAGAIN || errno == EWOULDBLOCK || errno == EINTR)) return;
    if (r <= 0) {               // closed before a full line: answer what there is
        on_line(c, c.inbuf);
        return;
    }
    c.inbuf.append(buf, (size_t)r);
    size_t nl = c.inbuf.find('\n');
    if (nl != std::string::npos) {
        on_line(c, c.inbuf.substr(0, nl));
    } else if (c.inbuf.size() >= kMaxLine) {
        answer(c, "ERR request line too long\n");
    }
}

void Daemon::on_line(Client &c, const std::string &line)
{
    c.line_ms = now_ms();
    c.req = parse_request(line);
    switch (c.req.verb) {
    case Verb::Ping:
        answer(c, "PONG 2\n");
        break;
    case Verb::Quit:
        answer(c, "BYE\n");
        quitting_ = true;
        break;
    case Verb::Decode:
        submit(c);
        break;
    case Verb::Malformed:
        answer(c, "ERR bad request\n");
        break;
    default:
        answer(c, "ERR unknown command\n");
        break;
    }
}

void Daemon::submit(Client &c)
{
    std::string err;
    std::vector<uint8_t> ogg;
    if (!read_file(c.req.in.c_str(), ogg, err)) return answer(c, "ERR " + err + "\n");
    char eb[512];
    int64_t play = 0, n16 = 0;
    int32_t ch = 0;
    if (cuopus_probe_pcm(ogg.data(), ogg.size(), &play, &ch, eb, sizeof eb)) return answer(c, std::string("ERR ") + eb + "\n");
    if (c.req.f16k) {
        if (ch != 1) return answer(c, "ERR only mono supported with DECODE16F\n");
        if (cuopus_probe(ogg.data(), ogg.size(), &n16, eb, sizeof eb)) return answer(c, std::string("ERR ") + eb + "\n");
        c.out_bytes = 4 * (size_t)n16;
    } else {
        c.out_bytes = 2 * (size_t)play * (size_t)ch;
    }
    c.play48 = play;
    c.srv = pool_.get(c.req, err);
    if (!c.srv) return answer(c, "ERR " + err + "\n");
    if (cuopus_server_submit(c.srv, ogg.data(), ogg.size(), &c.id, eb, sizeof eb))
        return answer(c, std::string("ERR ") + eb + "\n");
    c.host.resize(c.out_bytes ? c.out_bytes : 1);
    c.in_server = true;
    c.prep_ms = now_ms() - c.line_ms;
}

// Answer every submitted request the server has completed.
void Daemon::collect()
{
    for (Client &c : clients_) {
        if (!c.in_server) continue;
        int64_t nout = 0;
        int32_t ch = 0;
        double lat = 0;
        char eb[512];
        double t0 = now_ms();
        int rc = cuopus_server_wait(c.srv, c.id, 0, c.host.data(), c.host.size(), &nout, &ch, &lat, eb, sizeof eb);
        if (rc == 4) continue;   // still decoding
        double copy_ms = now_ms() - t0;
        c.in_server = false;
        if (rc) {
            answer(c, std::string("ERR ") + eb + "\n");
            continue;
        }
        std::string err;
        double t1 = now_ms();
        bool wrote = write_file(c.req.out.c_str(), c.host.data(), c.out_bytes, err);
        std::vector<uint8_t>().swap(c.host);
        if (!wrote) {
            answer(c, "ERR " + err + "\n");
            continue;
        }
        double write_ms = now_ms() - t1;
        unsigned long long values = c.req.f16k ? (unsigned long long)nout : (unsigned long long)nout * (unsigned)ch;
        char r[400];
        snprintf(r, sizeof r, "OK %llu %lld %.1f %.1f %.1f %.1f %.1f %.1f %.1f\n", values, c.play48, lat,
                 now_ms() - c.line_ms, c.prep_ms, 0.0, copy_ms, 0.0, write_ms);
        answer(c, r);
    }
}

int Daemon::run()
{
    if (!listen_on_path()) return 2;
    double t0 = now_ms();
    char eb[512];
    if (cuopus_warmup(eb, sizeof eb)) fprintf(stderr, "cuopus_decode: warmup: %s\n", eb);
    fprintf(stderr, "cuopus_decode: serving on %s (warmup %.0f ms, idle exit %ds)\n", path_.c_str(), now_ms() - t0,
            idle_s_);
    last_busy_ms_ = now_ms();
    for (;;) {
        bool busy = false;
        for (const Client &c : clients_) busy = busy || c.in_server;
        if (quitting_ && !busy) break;
        if (!clients_.empty()) last_busy_ms_ = now_ms();
        else if (now_ms() - last_busy_ms_ > idle_s_ * 1000.0) {
            fprintf(stderr, "cuopus_decode: idle %ds, exiting\n", idle_s_);
            break;
        }
        std::vector<struct pollfd> pf;
        if (!quitting_) pf.push_back({lfd_, POLLIN, 0});
        std::vector<size_t> who;
        for (size_t i = 0; i < clients_.size(); i++)
            if (!clients_[i].in_server && !clients_[i].done) {
                pf.push_back({clients_[i].fd, POLLIN, 0});
                who.push_back(i);
            }
        // decodes in flight: come back soon to collect them; otherwise wake at
        // least once a second for the line and idle timeouts
        int wait_ms = busy ? 2 : 1000;
        int pr = poll(pf.data(), pf.size(), wait_ms);
        if (pr < 0 && errno != EINTR) {
            perror("cuopus_decode: poll");
            break;
        }
        size_t base = quitting_ ? 0 : 1;
        if (pr > 0) {
            for (size_t k = 0; k < who.size(); k++)
                if (pf[base + k].revents & (POLLIN | POLLHUP | POLLERR)) on_readable(clients_[who[k]]);
            if (!quitting_ && (pf[0].revents & POLLIN)) {
                for (;;) {
                    int fd = accept(lfd_, nullptr, nullptr);
                    if (fd < 0) break;
                    Client c;
                    c.fd = fd;
                    c.accepted_ms = now_ms();
                    clients_.push_back(std::move(c));
                }
            }
        }
        collect();
        double now = now_ms();
        for (Client &c : clients_)
            if (!c.done && !c.in_server && now - c.accepted_ms > kLineTimeoutMs) answer(c, "ERR no request line\n");
        for (size_t i = 0; i < clients_.size();) {
            if (clients_[i].done) {
                close(clients_[i].fd);
                clients_.erase(clients_.begin() + (long)i);
            } else {
                i++;
            }
        }
    }
    for (Client &c : clients_) close(c.fd);
    clients_.clear();
    close(lfd_);
    unlink(path_.c_str());
    return 0;
}

// ------------------------------------------------------------------ command line
//
// Three modes: --serve <socket>, --ogg <in> [out|-] [options], and the legacy
// blob mode <packets.blob> <chains.bin> <out.pcm> [stride].  Options are read
// from one table; an argument that does not start with "--", or is "-",
// is positional.

struct CliArgs {
    std::vector<const char *> pos;
    double seg_s = 1.0, preroll_ms = DEF_PREROLL_MS;
    long stride = DEF_STRIDE;
    bool f16k = false, serve = false, ogg = false;
    const char *dump_blob = nullptr, *dump_chains = nullptr;
};

bool num(const char *v, double &out)
{
    char *end = nullptr;
    out = strtod(v, &end);
    return end != v && !*end;
}

// One entry per option: its name, whether it takes a value, and how it sets
// the arguments (false: the value does not parse).
struct OptSpec {
    const char *name;
    bool takes_value;
    bool (*apply)(CliArgs &, const char *);
};

const OptSpec kOpts[] = {
    {"--serve", false, [](CliArgs &a, const char *) { return a.serve = true; }},
    {"--ogg", false, [](CliArgs &a, const char *) { return a.ogg = true; }},
    {"--f16k", false, [](CliArgs &a, const char *) { return a.f16k = true; }},
    {"--seg", true, [](CliArgs &a, const char *v) { return num(v, a.seg_s); }},
    {"--preroll", true, [](CliArgs &a, const char *v) { return num(v, a.preroll_ms); }},
    {"--stride", true,
     [](CliArgs &a, const char *v) {
         double d = 0;
         bool ok = num(v, d);
         a.stride = (long)d;
         return ok;
     }},
    {"--dump-blob", true, [](CliArgs &a, const char *v) { return (a.dump_blob = v) != nullptr; }},
    {"--dump-chains", true, [](CliArgs &a, const char *v) { return (a.dump_chains = v) != nullptr; }},
};

bool parse_args(int argc, char **argv, CliArgs &a, std::string &err)
{
    for (int i = 1; i < argc; i++) {
        const char *s = argv[i];
        if (strncmp(s, "--", 2) != 0) {
            a.pos.push_back(s);
            continue;
        }
        const OptSpec *o = nullptr;
        for (const OptSpec &c : kOpts)
            if (!strcmp(c.name, s)) o = &c;
        if (!o) {
            err = std::string("unknown option ") + s;
            return false;
        }
        const char *v = nullptr;
        if (o->takes_value) {
            if (i + 1 >= argc) {
                err = std::string(s) + " needs a value";
                return false;
            }
            v = argv[++i];
        }
        if (!o->apply(a, v)) {
            err = std::string("bad value for ") + s + ": " + (v ? v : "");
            return false;
        }
    }
    if (a.stride < 1) a.stride = 1;
    return true;
}

int usage(const char *prog)
{
    fprintf(stderr,
            "usage: %s <packets.blob> <chains.bin> <out.pcm> [stride]\n"
            "       %s --ogg <in.ogg> [out.pcm|-] [--seg S] [--preroll MS] [--stride N] [--f16k]\n"
            "                 [--dump-blob F] [--dump-chains F]\n"
            "       %s --serve <unix_socket>\n",
            prog, prog, prog);
    return 2;
}

} // namespace

int main(int argc, char **argv)
{
    CliArgs a;
    std::string err;
    if (!parse_args(argc, argv, a, err)) {
        fprintf(stderr, "cuopus_decode: %s\n", err.c_str());
        return 2;
    }
    if (a.serve) {
        if (a.pos.size() != 1) return usage(argv[0]);
        int idle_s = 600;
        if (const char *e = getenv("CUOPUS_SERVE_IDLE_S"))
            if (atoi(e) > 0) idle_s = atoi(e);
        Daemon d(a.pos[0], idle_s);
        return d.run();
    }
    if (a.ogg) {
        if (a.pos.empty() || a.pos.size() > 2) return usage(argv[0]);
        return run_ogg_once(a.pos[0], a.pos.size() > 1 ? a.pos[1] : nullptr, a.seg_s, a.preroll_ms,
                            (unsigned)a.stride, a.f16k, a.dump_blob, a.dump_chains);
    }
    if (a.pos.size() < 3 || a.pos.size() > 4) return usage(argv[0]);
    unsigned stride = DEF_STRIDE;
    if (a.pos.size() == 4) {
        long v = strtol(a.pos[3], nullptr, 10);
        stride = (unsigned)(v < 1 ? 1 : v);
    }
    return run_blob(a.pos[0], a.pos[1], a.pos[2], stride);
}
