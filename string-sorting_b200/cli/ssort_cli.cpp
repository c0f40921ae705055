// ssort_cli.cpp -- command-line front end for whole-file inputs: reads a file
// straight into pinned host memory, finds and sorts its strings on the GPU the
// way the reference's sortstring makes them (lines by default, NUL-delimited
// with --raw, every suffix with --suffix-sorting; src/sortstring.c:310-358),
// and optionally checks the order (--check, the test of src/util/debug.h:42-72)
// and writes the sorted strings one per line (--write, src/sortstring.c:361-384).
//
//   ssort-sort [--raw] [--suffix-sorting] [--check] [--write FILE] [--device N] FILE
#include "ssort_b200.h"

#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace {

[[noreturn]] void die(const std::string &msg) {
    std::fprintf(stderr, "ERROR: %s\n", msg.c_str());
    std::exit(1);
}

void check_status(int rc, const char *what) {
    if (rc != SSORT_OK)
        die(std::string(what) + ": " + ssort_strerror(rc) + ": " + ssort_last_error());
}

void usage() {
    std::fprintf(stderr,
                 "usage: ssort-sort [--raw] [--suffix-sorting] [--check] [--write FILE] "
                 "[--device N] FILE\n");
    std::exit(2);
}

}  // namespace

int main(int argc, char **argv) {
    int mode = SSORT_TEXT_LINES;
    bool check = false;
    const char *write_path = nullptr;
    const char *path = nullptr;
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--raw")
            mode = SSORT_TEXT_RAW;
        else if (a == "--suffix-sorting")
            mode = SSORT_TEXT_SUFFIXES;
        else if (a == "--check")
            check = true;
        else if (a == "--write" && i + 1 < argc)
            write_path = argv[++i];
        else if (a == "--device" && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else if (!a.empty() && a[0] == '-')
            usage();
        else
            path = argv[i];
    }
    if (!path) usage();

    const int fd = open(path, O_RDONLY);
    if (fd < 0) die(std::string("unable to open '") + path + "': " + std::strerror(errno));
    struct stat sb;
    if (fstat(fd, &sb) != 0 || sb.st_size <= 0)
        die(std::string("input file '") + path + "' empty or unreadable");
    const size_t len = (size_t)sb.st_size;
    unsigned char *text = nullptr;
    check_status(ssort_pinned_alloc(len + 16, (void **)&text), "pinned allocation");
    for (size_t got = 0; got < len;) {
        const ssize_t r = read(fd, text + got, std::min<size_t>(len - got, 1u << 24));
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) die(std::string("read failed on '") + path + "'");
        got += (size_t)r;
    }
    close(fd);
    std::memset(text + len, 0, 16);

    ssort_ctx *ctx = nullptr;
    check_status(ssort_ctx_create(device, &ctx), "context");
    uint64_t n = 0;
    if (mode == SSORT_TEXT_SUFFIXES) {
        n = len;
    } else {
        const unsigned char delim = mode == SSORT_TEXT_LINES ? '\n' : 0;
        for (size_t i = 0; i < len; ++i) n += text[i] == delim;
    }
    if (n == 0) die("unable to read any strings from the input file");
    std::vector<uint64_t> sorted(n);
    const auto t0 = std::chrono::steady_clock::now();
    uint64_t got_n = 0;
    check_status(ssort_sort_text_host(ctx, text, len, mode, sorted.data(), nullptr, n, &got_n),
                 "sort");
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (got_n != n) die("string count mismatch");
    std::fprintf(stderr, "sorted %llu strings of %zu bytes in %.3f ms\n", (unsigned long long)n,
                 len, ms);

    // The strings as the reference sees them: '\n' delimiters become NUL.
    if (mode == SSORT_TEXT_LINES)
        for (size_t i = 0; i < len; ++i)
            if (text[i] == '\n') text[i] = 0;
    int rc = 0;
    if (check) {
        size_t wrong = 0, identical = 0;
        for (uint64_t k = 0; k + 1 < n; ++k) {
            if (sorted[k] == sorted[k + 1]) ++identical;
            if (std::strcmp((const char *)text + sorted[k], (const char *)text + sorted[k + 1]) > 0)
                ++wrong;
        }
        if (identical) std::fprintf(stderr, "WARNING: found %zu identical pointers!\n", identical);
        if (wrong) std::fprintf(stderr, "WARNING: found %zu incorrect orderings!\n", wrong);
        std::fprintf(stderr, "Checking: %s\n", (wrong || identical) ? "BAD" : "GOOD");
        rc = (wrong || identical) ? 1 : 0;
    }
    if (write_path) {
        FILE *fp = std::fopen(write_path, "w");
        if (!fp) die(std::string("unable to open '") + write_path + "' for writing");
        for (uint64_t k = 0; k < n; ++k) {
            std::fputs((const char *)text + sorted[k], fp);
            std::fputc('\n', fp);
        }
        std::fclose(fp);
    }
    ssort_ctx_destroy(ctx);
    ssort_pinned_free(text);
    return rc;
}
