// p2g_cli.cpp -- `par2rust create` over the C ABI (the CLI of src/main.rs):
//
//   par2rust create|c [-s SIZE] [-c N | -r PCT|[gmk]N] [--single-volume]
//                     [-u] [-l] [-n N] [-t N] [-o PATH] [--comment TEXT]...
//                     [-R] [-i PATH|-] [-q] [ARCHIVE] INPUTS...
//
// Positionals: without --out the first one is the archive (src/main.rs:
// 195-222).  Inputs come from the positionals and --input-file (one path per
// line, blank lines and '#' lines skipped, :226-247); directories need
// --recurse (:252-279).  Every input is scanned (p2g_scan) before anything
// is written; -r resolves against the scanned slice count, the volume
// scheme follows the flags (p2g_build_volume_scheme), and the create runs
// through p2g_run_create.  Errors print "par2rust: error: <message>" and exit
// with status 1.  -t is accepted for compatibility (host threads are the
// library's own).  Progress bars are not drawn; without -q the written files
// are listed as the reference prints them.
#include <dirent.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/par2gpu.h"

namespace {

struct Args {
    uint64_t slice_size = 4096;
    uint32_t recovery_count = 0;
    bool has_count = false, has_redundancy = false;
    p2g_redundancy redundancy{};
    p2g_cli_volume_flags vol{};
    std::string out;
    bool has_out = false;
    std::vector<std::string> comments;
    bool recurse = false, quiet = false;
    std::string input_file;
    bool has_input_file = false;
    std::vector<std::string> positionals;
};

struct Failure {
    std::string msg;
};

[[noreturn]] void fail(const std::string& m) { throw Failure{m}; }
[[noreturn]] void fail_status() { throw Failure{p2g_last_error_message()}; }

std::string io_error(int err) { return std::string("I/O error: ") + strerror(err) + " (os error " + std::to_string(err) + ")"; }

void usage_exit(const char* what) {
    fprintf(stderr,
            "par2rust: error: %s\n\nUsage: par2rust create [OPTIONS] [POSITIONALS]...\n"
            "  -s, --slice-size <SIZE>      block size, bytes or with a b/k/m/g suffix [default: 4096]\n"
            "  -c, --recovery-count <N>     recovery blocks [default: 0]\n"
            "  -r, --redundancy <PCT|[gmk]N> percent of the input, or a target size\n"
            "      --single-volume          one vol0+N file\n"
            "  -u, --uniform                uniform volumes (-n sets their count)\n"
            "  -l, --limit-size             cap volumes at the largest source file\n"
            "  -n, --volume-count <N>       number of volumes (with -u)\n"
            "  -t, --threads <N>            accepted for compatibility\n"
            "  -o, --out <PATH>             archive name; all positionals are inputs\n"
            "      --comment <TEXT>         comment packet (repeatable)\n"
            "  -R, --recurse                walk directory inputs\n"
            "  -i, --input-file <PATH>      more inputs, one per line ('-' = stdin)\n"
            "  -q, --quiet                  no summary\n",
            what);
    exit(2);
}

uint32_t parse_u32(const std::string& flag, const std::string& v) {
    char* end = nullptr;
    errno = 0;
    const unsigned long long x = strtoull(v.c_str(), &end, 10);
    if (v.empty() || *end || errno || x > 0xFFFFFFFFull || v[0] == '-')
        usage_exit(("invalid value '" + v + "' for '" + flag + "'").c_str());
    return (uint32_t)x;
}

Args parse_args(int argc, char** argv) {
    Args a;
    if (argc < 2) usage_exit("a subcommand is required: create (alias c)");
    const std::string cmd = argv[1];
    if (cmd == "-h" || cmd == "--help") usage_exit("usage");
    if (cmd != "create" && cmd != "c") usage_exit(("unrecognized subcommand '" + cmd + "'").c_str());
    bool only_positionals = false;
    for (int i = 2; i < argc; ++i) {
        std::string t = argv[i];
        if (only_positionals || t == "-" || t.empty() || t[0] != '-') {
            a.positionals.push_back(t);
            continue;
        }
        if (t == "--") {
            only_positionals = true;
            continue;
        }
        std::string name, value;
        bool has_value = false;
        if (t.rfind("--", 0) == 0) {
            const size_t eq = t.find('=');
            name = t.substr(0, eq);
            if (eq != std::string::npos) {
                value = t.substr(eq + 1);
                has_value = true;
            }
        } else {
            name = t.substr(0, 2);
            if (t.size() > 2) {
                value = t.substr(2);
                has_value = true;
            }
        }
        auto take = [&]() -> std::string {
            if (has_value) return value;
            if (i + 1 >= argc) usage_exit(("a value is required for '" + name + "'").c_str());
            return std::string(argv[++i]);
        };
        auto flag = [&]() {
            if (has_value) usage_exit(("unexpected value for '" + name + "'").c_str());
        };
        if (name == "-s" || name == "--slice-size") {
            if (p2g_parse_slice_size(take().c_str(), &a.slice_size) != P2G_OK)
                usage_exit(p2g_last_error_message());
        } else if (name == "-c" || name == "--recovery-count") {
            a.recovery_count = parse_u32(name, take());
            a.has_count = true;
        } else if (name == "-r" || name == "--redundancy") {
            if (p2g_parse_redundancy(take().c_str(), &a.redundancy) != P2G_OK) usage_exit(p2g_last_error_message());
            a.has_redundancy = true;
        } else if (name == "--single-volume") {
            flag();
            a.vol.single_volume = 1;
        } else if (name == "-u" || name == "--uniform") {
            flag();
            a.vol.uniform = 1;
        } else if (name == "-l" || name == "--limit-size") {
            flag();
            a.vol.limit_size = 1;
        } else if (name == "-n" || name == "--volume-count") {
            a.vol.volume_count = parse_u32(name, take());
            a.vol.has_volume_count = 1;
        } else if (name == "-t" || name == "--threads") {
            parse_u32(name, take());
        } else if (name == "-o" || name == "--out") {
            a.out = take();
            a.has_out = true;
        } else if (name == "--comment") {
            a.comments.push_back(take());
        } else if (name == "-R" || name == "--recurse") {
            flag();
            a.recurse = true;
        } else if (name == "-i" || name == "--input-file") {
            a.input_file = take();
            a.has_input_file = true;
        } else if (name == "-q" || name == "--quiet") {
            flag();
            a.quiet = true;
        } else if (name == "-h" || name == "--help") {
            usage_exit("usage");
        } else {
            usage_exit(("unexpected argument '" + t + "'").c_str());
        }
    }
    if (a.has_count && a.has_redundancy)
        usage_exit("the argument '--redundancy <PCT|[gmk]N>' cannot be used with '--recovery-count <RECOVERY_COUNT>'");
    return a;
}

// read_input_file_list, src/main.rs:226-247
std::vector<std::string> read_list(const std::string& path) {
    std::vector<std::string> out;
    std::ifstream f;
    std::istream* in = &std::cin;
    if (path != "-") {
        f.open(path);
        if (!f) fail(io_error(errno ? errno : ENOENT));
        in = &f;
    }
    std::string line;
    while (std::getline(*in, line)) {
        size_t b = 0, e = line.size();
        while (b < e && isspace((unsigned char)line[b])) ++b;
        while (e > b && isspace((unsigned char)line[e - 1])) --e;
        line = line.substr(b, e - b);
        if (!line.empty() && line[0] != '#') out.push_back(line);
    }
    return out;
}

// depth-first walk in directory order, regular files only, symlinks not followed
void walk(const std::string& dir, std::vector<std::string>& out) {
    DIR* d = opendir(dir.c_str());
    if (!d) fail(io_error(errno));
    std::vector<std::string> entries;
    while (dirent* e = readdir(d)) {
        const std::string n = e->d_name;
        if (n != "." && n != "..") entries.push_back(n);
    }
    closedir(d);
    for (const std::string& n : entries) {
        const std::string p = dir + "/" + n;
        struct stat st;
        if (lstat(p.c_str(), &st) != 0) fail(io_error(errno));
        if (S_ISDIR(st.st_mode))
            walk(p, out);
        else if (S_ISREG(st.st_mode))
            out.push_back(p);
    }
}

// expand_input_paths, src/main.rs:252-279
std::vector<std::string> expand(const std::vector<std::string>& raw, bool recurse) {
    std::vector<std::string> out;
    for (const std::string& p : raw) {
        struct stat st;
        if (stat(p.c_str(), &st) != 0) fail(io_error(errno));
        if (S_ISDIR(st.st_mode)) {
            if (!recurse)
                fail("I/O error: input \"" + p + "\" is a directory; pass --recurse to walk it recursively");
            walk(p, out);
        } else {
            out.push_back(p);
        }
    }
    return out;
}

// display_name_for, src/main.rs:448-454: the basename
std::string display_name(const std::string& p) {
    std::string s = p;
    while (s.size() > 1 && s.back() == '/') s.pop_back();
    const size_t k = s.rfind('/');
    const std::string base = k == std::string::npos ? s : s.substr(k + 1);
    return base.empty() || base == "." || base == ".." ? p : base;
}

int run(int argc, char** argv) {
    Args a = parse_args(argc, argv);
    std::string output;
    std::vector<std::string> raw;
    if (a.has_out) {
        output = a.out;
        raw = a.positionals;
    } else {
        if (a.positionals.empty())
            fail("I/O error: missing output archive: pass it as the first positional argument or use --out PATH");
        output = a.positionals[0];
        raw.assign(a.positionals.begin() + 1, a.positionals.end());
    }
    if (a.has_input_file) {
        std::vector<std::string> more = read_list(a.input_file);
        raw.insert(raw.end(), more.begin(), more.end());
    }
    const std::vector<std::string> inputs = expand(raw, a.recurse);
    if (inputs.empty()) fail("no input files supplied");

    std::vector<p2g_source_file> sources(inputs.size());
    uint64_t total_blocks = 0, largest = 0;
    for (size_t i = 0; i < inputs.size(); ++i) {
        const std::string name = display_name(inputs[i]);
        if (p2g_scan(inputs[i].c_str(), (const uint8_t*)name.data(), name.size(), a.slice_size, &sources[i]) != P2G_OK) {
            const std::string m = p2g_last_error_message();
            for (size_t k = 0; k < i; ++k) p2g_source_file_free(&sources[k]);
            fail(m);
        }
        total_blocks += sources[i].slice_count;
        if (sources[i].length > largest) largest = sources[i].length;
    }
    auto release = [&]() {
        for (auto& s : sources) p2g_source_file_free(&s);
    };
    uint32_t R = a.recovery_count;
    if (a.has_redundancy && p2g_resolve_redundancy(&a.redundancy, total_blocks, a.slice_size, &R) != P2G_OK) {
        release();
        fail_status();
    }
    if (R > P2G_MAX_RECOVERY_BLOCKS) {
        release();
        fail("recovery block count " + std::to_string(R) + " exceeds PAR2 limit of 65535");
    }
    p2g_volume_scheme scheme, inner;
    if (p2g_build_volume_scheme(&a.vol, largest, a.slice_size, R, &scheme, &inner) != P2G_OK) {
        release();
        fail_status();
    }
    std::vector<const char*> cm;
    for (const std::string& c : a.comments) cm.push_back(c.c_str());
    p2g_create_options opts;
    memset(&opts, 0, sizeof opts);
    opts.output = output.c_str();
    opts.slice_size = a.slice_size;
    opts.recovery_block_count = R;
    opts.volume_scheme = scheme;
    opts.comments = cm.empty() ? nullptr : cm.data();
    opts.comment_count = (uint32_t)cm.size();
    p2g_path_list written{};
    const p2g_status st = p2g_run_create(&opts, sources.data(), (uint32_t)sources.size(), &written);
    release();
    if (st != P2G_OK) fail_status();
    if (!a.quiet) {
        printf("Wrote %u file%s:\n", written.count, written.count == 1 ? "" : "s");
        for (uint32_t i = 0; i < written.count; ++i) {
            struct stat s;
            const long long size = stat(written.paths[i], &s) == 0 ? (long long)s.st_size : 0;
            printf("  %s (%lld bytes)\n", written.paths[i], size);
        }
    }
    p2g_path_list_free(&written);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const Failure& f) {
        fprintf(stderr, "par2rust: error: %s\n", f.msg.c_str());
        return 1;
    }
}
