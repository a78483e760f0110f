// pi_b200 -- command-line program with the reference's pi_compute flags (src/main.cpp:25-105)
// plus the B200 modes.
//
//   pi_b200 --digits N [--output FILE] [--threads T] [--verbose]
//           [--gpu | --b200]           products >= --gpu-threshold limbs on the B200, per call
//           [--batched]                the whole computation in HBM: level-batched binary splitting,
//                                      Newton finish and batched decimal conversion on the device
//           [--host-finish]            batched splitting on the device, Newton finish and conversion on
//                                      the host with B200 products
//           [--newton | --mpf]         final formula + radix conversion: Newton iterations and divide-
//                                      and-conquer conversion on B200 products, or the reference's GMP mpf
//           [--gpu-threshold N]        (default 10000 like the reference)
//           [--device D]
//           [--checkpoint DIR]         with --batched: resume from and save the reference's checkpoint
//                                      files (bs_<a>_<b>.ckpt, pi_int_<N>.ckpt) in DIR
//           [--resume]                 accepted like the reference's flag; checkpoints found in DIR are
//                                      always used, as in the reference (src/main.cpp:94-97)
#include <fcntl.h>
#include <sys/mman.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>

#include "b200_multiplier.h"
#include "pi_engine.h"

// The output file mapped for writing, its pages touched, so that the device's digits are copied
// straight into the page cache: no 100 MB string to fill and no second copy by fwrite. Made on a
// thread while the device context is created. Not used (fwrite instead) where the file cannot be
// mapped, e.g. a pipe.
struct OutputMap {
    int fd = -1;
    char* p = nullptr;
    size_t n = 0;
    void open_map(const std::string& path, size_t bytes) {
        fd = ::open(path.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0644);
        if (fd < 0) return;
        void* m = MAP_FAILED;
        if (::ftruncate(fd, (off_t)bytes) == 0) m = ::mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
        if (m == MAP_FAILED) {
            ::close(fd);
            fd = -1;
            return;
        }
        p = static_cast<char*>(m);
        n = bytes;
        const long pg = ::sysconf(_SC_PAGESIZE);
        for (size_t i = 0; i < bytes; i += (size_t)(pg > 0 ? pg : 4096)) p[i] = '0';
    }
    // Unmaps and closes; false on an error (the file is then not trusted).
    bool finish() {
        bool ok = true;
        if (p) ok = ::munmap(p, n) == 0;
        if (fd >= 0) ok = (::close(fd) == 0) && ok;
        p = nullptr;
        fd = -1;
        return ok;
    }
};

static void usage() {
    std::puts(
        "pi_b200 - pi digits with exact big-integer products on one B200\n\n"
        "USAGE: pi_b200 --digits <N> [--output FILE] [--threads T] [--gpu|--b200] [--batched|--host-finish]\n"
        "               [--newton|--mpf]\n"
        "               [--gpu-threshold N] [--device D] [--checkpoint DIR [--resume]] [--verbose]\n");
}

int main(int argc, char** argv) {
    const auto t_main = std::chrono::steady_clock::now();
    const auto wall_main = std::chrono::system_clock::now();
    // Load every kernel when the CUDA context is created (unless the caller chose otherwise): a run
    // uses most of them, and loading them one by one at first launch costs this one-shot process
    // more (measured on a B200: the twiddle-table build 49 -> 6 ms, the first pi run 10-20 ms less).
    setenv("CUDA_MODULE_LOADING", "EAGER", 0);
    pi::PiConfig cfg;
    bool has_digits = false, gpu = false, resume = false;
    size_t threshold = 10000;
    std::string output = "pi_digits.txt";
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--help" || a == "-h") {
            usage();
            return 0;
        } else if (a == "--digits" && i + 1 < argc) {
            cfg.digits = std::stoul(argv[++i]);
            has_digits = true;
        } else if (a == "--output" && i + 1 < argc) {
            output = argv[++i];
        } else if (a == "--threads" && i + 1 < argc) {
            cfg.num_threads = std::stoul(argv[++i]);
        } else if (a == "--gpu" || a == "--b200" || a == "--ntt") {
            gpu = true;
        } else if (a == "--batched") {
            cfg.mode = pi::BSMode::Batched;
            cfg.final_mode = pi::FinalMode::Device;
        } else if (a == "--host-finish") {
            cfg.mode = pi::BSMode::Batched;
            cfg.final_mode = pi::FinalMode::Newton;
        } else if (a == "--newton") {
            cfg.final_mode = pi::FinalMode::Newton;
        } else if (a == "--mpf") {
            cfg.final_mode = pi::FinalMode::Mpf;
        } else if (a == "--gpu-threshold" && i + 1 < argc) {
            threshold = std::stoul(argv[++i]);
        } else if (a == "--device" && i + 1 < argc) {
            cfg.device = std::stoi(argv[++i]);
        } else if (a == "--checkpoint" && i + 1 < argc) {
            cfg.checkpoint_dir = argv[++i];
        } else if (a == "--resume") {
            resume = true;
        } else if (a == "--verbose" || a == "-v") {
            cfg.verbose = true;
        } else {
            std::fprintf(stderr, "Unknown option: %s\n", a.c_str());
            usage();
            return 1;
        }
    }
    if (!has_digits || cfg.digits == 0) {
        std::fprintf(stderr, "Error: --digits <N> (N > 0) is required\n");
        return 1;
    }
    if (resume && cfg.checkpoint_dir.empty()) {
        std::fprintf(stderr, "Error: --resume requires --checkpoint <DIR>\n");
        return 1;
    }
    if (!cfg.checkpoint_dir.empty() &&
        !(cfg.mode == pi::BSMode::Batched && cfg.final_mode == pi::FinalMode::Device)) {
        std::fprintf(stderr, "Error: --checkpoint needs --batched (the device-resident pipeline)\n");
        return 1;
    }
    std::string mapped;  // the output file while it holds no digits yet (removed on an error)
    try {
        // The device context (CUDA context, twiddle tables, tuned splits) is made first so that the
        // trace can report it apart from the computation.
        const auto t_ctx = std::chrono::steady_clock::now();
        const bool device_digits = cfg.mode == pi::BSMode::Batched && cfg.final_mode == pi::FinalMode::Device;
        OutputMap om;
        std::thread mapper;
        if (device_digits) mapper = std::thread([&om, &output, &cfg] { om.open_map(output, cfg.digits + 2); });
        struct Joiner {
            std::thread& t;
            ~Joiner() {
                if (t.joinable()) t.join();
            }
        } joiner{mapper};
        pg_ctx* dev_ctx = (cfg.mode == pi::BSMode::Batched || gpu) ? pi::shared_context(cfg.device) : nullptr;
        std::unique_ptr<pi::Multiplier> mult;
        const char* mode = "CPU";
        if (gpu && cfg.mode == pi::BSMode::PerCall) {
            mult = std::make_unique<pi::B200Multiplier>(threshold, dev_ctx, cfg.device);
            mode = "B200 per-call";
        } else {
            mult = std::make_unique<pi::GmpMultiplier>();
            if (cfg.mode == pi::BSMode::Batched) mode = "B200 batched";
        }
        pi::PiEngine eng(*mult);
        if (mapper.joinable()) mapper.join();
        cfg.digits_out = om.p;
        if (om.p) mapped = output;
        const auto t_compute = std::chrono::steady_clock::now();
        pi::PiResult r = eng.compute(cfg);
        const auto t_write = std::chrono::steady_clock::now();
        if (om.p) {
            if (!om.finish()) throw std::runtime_error("cannot write " + output);
            mapped.clear();
        } else {
            om.finish();
            FILE* f = std::fopen(output.c_str(), "wb");
            if (!f) throw std::runtime_error("cannot open " + output);
            const bool written = std::fwrite(r.digits.data(), 1, r.digits.size(), f) == r.digits.size();
            if (std::fclose(f) != 0 || !written) throw std::runtime_error("cannot write " + output);
        }
        if (cfg.verbose || std::getenv("PI_B200_TRACE")) {
            auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            const auto t_end = std::chrono::steady_clock::now();
            std::printf("  Process: main %.1f ms, device context %.1f ms, compute %.1f ms, file %.1f ms\n",
                        ms(t_main, t_ctx), ms(t_ctx, t_compute), ms(t_compute, t_write), ms(t_write, t_end));
        }
        std::printf("Computed %zu digits of pi in %g seconds (%lu terms, %s).\nOutput written to: %s\n", cfg.digits,
                    r.elapsed_seconds, r.terms_used, mode, output.c_str());
        if (auto* b = dynamic_cast<pi::B200Multiplier*>(mult.get())) {
            if (cfg.verbose) b->print_stats();
        }
        // The output file is closed and checked: leave without tearing the device context down
        // (freeing gigabytes of device buffers one by one takes longer than the driver's own
        // clean-up of an exiting process).
        if (cfg.verbose || std::getenv("PI_B200_TRACE")) {
            // wall-clock stamps of main's entry and of the exit, for a caller that splits its own
            // measurement of the process into start-up, the timed parts and the exit
            auto ns = [](std::chrono::system_clock::time_point t) {
                return (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(t.time_since_epoch()).count();
            };
            std::printf("  Clock: main %lld ns, exit %lld ns\n", ns(wall_main), ns(std::chrono::system_clock::now()));
        }
        std::fflush(stdout);
        std::fflush(stderr);
        _exit(0);
    } catch (const std::exception& e) {
        if (!mapped.empty()) ::unlink(mapped.c_str());  // no file of zeros left behind
        std::fprintf(stderr, "Error: %s\n", e.what());
        return 1;
    }
}
