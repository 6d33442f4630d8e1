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

void reply(int fd, const std::string &msg)
{
    size_t o = 0;
    while (o < msg.size()) {
        ssize_t w = write(fd, msg.data() + o, msg.size() - o);
        if (w <= 0) break;
        o += (size_t)w;
    }
}

int run_serve(const char *sock_path)
{
    signal(SIGPIPE, SIG_IGN);
    int idle_s = 600;
    const char *e = getenv("CUOPUS_SERVE_IDLE_S");
    if (e && atoi(e) > 0) idle_s = atoi(e);
    struct sockaddr_un addr;
    if (strlen(sock_path) >= sizeof(addr.sun_path)) {
        fprintf(stderr, "cuopus_decode: socket path longer than %zu bytes\n", sizeof(addr.sun_path) - 1);
        return 2;
    }
    unlink(sock_path);
    int srv = socket(AF_UNIX, SOCK_STREAM, 0);
    if (srv < 0) {
        perror("socket");
        return 2;
    }
    memset(&addr, 0, sizeof addr);
    addr.sun_family = AF_UNIX;
    strncpy(addr.sun_path, sock_path, sizeof(addr.sun_path) - 1);
    if (bind(srv, (struct sockaddr *)&addr, sizeof addr) < 0) {
        perror("bind");
        return 2;
    }
    if (listen(srv, 16) < 0) {
        perror("listen");
        return 2;
    }
    double t0 = now_ms();
    char eb[512];
    if (cuopus_warmup(eb, sizeof eb)) fprintf(stderr, "cuopus_decode: warmup: %s\n", eb);
    fprintf(stderr, "cuopus_decode: serving on %s (warmup %.0f ms, idle exit %ds)\n", sock_path, now_ms() - t0,
            idle_s);
    std::vector<char> line(8192);
    for (;;) {
        struct pollfd pfd = {srv, POLLIN, 0};
        int pr = poll(&pfd, 1, idle_s * 1000);
        if (pr == 0) {
            fprintf(stderr, "cuopus_decode: idle %ds, exiting\n", idle_s);
            unlink(sock_path);
            return 0;
        }
        if (pr < 0) {
            if (errno == EINTR) continue;
            perror("poll");
            return 2;
        }
        int fd = accept(srv, nullptr, nullptr);
        if (fd < 0) continue;
        // A client that connects and sends no request line must not hold the
        // single-threaded loop: its read gives up after 30 s.
        struct timeval rto = {30, 0};
        setsockopt(fd, SOL_SOCKET, SO_RCVTIMEO, &rto, sizeof rto);
        size_t got = 0;
        while (got < line.size() - 1) {
            ssize_t r = read(fd, line.data() + got, line.size() - 1 - got);
            if (r <= 0) break;
            got += (size_t)r;
            if (memchr(line.data(), '\n', got)) break;
        }
        line[got] = 0;
        char *nl = strchr(line.data(), '\n');
        if (nl) *nl = 0;
        const char *ln = line.data();
        int mode16 = -1;
        const char *args = nullptr;
        if (!strncmp(ln, "DECODE16F ", 10)) {
            mode16 = 1;
            args = ln + 10;
        } else if (!strncmp(ln, "DECODE ", 7)) {
            mode16 = 0;
            args = ln + 7;
        }
        if (!strncmp(ln, "PING", 4)) {
            reply(fd, "PONG 2\n");
        } else if (!strncmp(ln, "QUIT", 4)) {
            reply(fd, "BYE\n");
            close(fd);
            unlink(sock_path);
            return 0;
        } else if (mode16 >= 0) {
            double seg_s = 0, preroll_ms = 0;
            unsigned stride = DEF_STRIDE;
            std::vector<char> ogg(4096), out(4096);
            if (sscanf(args, "%lf %lf %u %4095s %4095s", &seg_s, &preroll_ms, &stride, ogg.data(), out.data()) != 5) {
                reply(fd, "ERR bad request\n");
            } else {
                double rt0 = now_ms();
                std::string err;
                std::vector<uint8_t> data;
                Report rep;
                int rc = read_file(ogg.data(), data, err) ? 0 : 2;
                double read_ms = now_ms() - rt0;
                if (!rc) {
                    set_env_params(seg_s, preroll_ms, stride);
                    rc = decode_ogg(data, out.data(), mode16 == 1, rep, err);
                }
                if (!rc) {
                    char r[400];
                    snprintf(r, sizeof r, "OK %llu %lld %.1f %.1f %.1f %.1f %.1f %.1f %.1f\n", rep.out_samples,
                             rep.play48, rep.st.kernel_ms, now_ms() - rt0, read_ms + rep.st.demux_ms,
                             rep.st.h2d_ms, rep.d2h_ms, rep.st.resample_ms, rep.fwrite_ms);
                    reply(fd, r);
                } else {
                    reply(fd, "ERR " + err + "\n");
                }
            }
        } else {
            reply(fd, "ERR unknown command\n");
        }
        close(fd);
    }
}

} // namespace

int main(int argc, char **argv)
{
    if (argc >= 3 && !strcmp(argv[1], "--serve")) return run_serve(argv[2]);
    if (argc >= 3 && !strcmp(argv[1], "--ogg")) {
        const char *ogg = argv[2];
        const char *out = nullptr, *dump_blob = nullptr, *dump_chains = nullptr;
        double seg_s = 1.0, preroll_ms = DEF_PREROLL_MS;
        unsigned stride = DEF_STRIDE;
        bool f16k = false;
        int ai = 3;
        if (ai < argc && (argv[ai][0] != '-' || !strcmp(argv[ai], "-"))) out = argv[ai++];
        for (; ai < argc; ai++) {
            if (!strcmp(argv[ai], "--seg") && ai + 1 < argc) seg_s = atof(argv[++ai]);
            else if (!strcmp(argv[ai], "--preroll") && ai + 1 < argc) preroll_ms = atof(argv[++ai]);
            else if (!strcmp(argv[ai], "--stride") && ai + 1 < argc) stride = (unsigned)atoi(argv[++ai]);
            else if (!strcmp(argv[ai], "--f16k")) f16k = true;
            else if (!strcmp(argv[ai], "--dump-blob") && ai + 1 < argc) dump_blob = argv[++ai];
            else if (!strcmp(argv[ai], "--dump-chains") && ai + 1 < argc) dump_chains = argv[++ai];
            else {
                fprintf(stderr, "cuopus_decode: unknown option %s\n", argv[ai]);
                return 2;
            }
        }
        if (stride < 1) stride = 1;
        return run_ogg_once(ogg, out, seg_s, preroll_ms, stride, f16k, dump_blob, dump_chains);
    }
    if (argc < 4) {
        fprintf(stderr,
                "usage: %s <packets.blob> <chains.bin> <out.pcm> [stride]\n"
                "       %s --ogg <in.ogg> [out.pcm|-] [--seg S] [--preroll MS] [--stride N] [--f16k]\n"
                "                 [--dump-blob F] [--dump-chains F]\n"
                "       %s --serve <unix_socket>\n",
                argv[0], argv[0], argv[0]);
        return 2;
    }
    unsigned stride = argc > 4 ? (unsigned)atoi(argv[4]) : DEF_STRIDE;
    if (stride < 1) stride = 1;
    return run_blob(argv[1], argv[2], argv[3], stride);
}
