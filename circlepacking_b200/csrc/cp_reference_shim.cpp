// Drop-in definitions of the reference's argument-less driver functions on top
// of the C ABI, so that the reference's prover.cpp (which declares
// circlepacking::lane_packing::find_critical_intervals() and calls
// algcuda::device::set_printf_buffer_size) links against this library unchanged.
//
//   lane_packing.cu:32-37            find_critical_intervals()
//   start_configuration.cu:217-225   find_critical_intervals_start_configuration()
//   start_configuration.cu:300-308   find_critical_intervals_start_end_configuration()
//   middle_configuration.cu:207-212  find_critical_intervals_middle_configuration()
//   end_configuration.cu:270-286     find_critical_intervals_end_configuration()
//   run_kernel.cuh:36-132            the lambda loop and its SIGINT handling
//
// Each family runs cp_prove_family_reference over [lambda_min, lambda_max] with
// the reference's lattice sizes, printing "Handling lambda interval [lb, ub]" to
// stderr before every launch as run_kernel.cuh:79 does.  On SIGINT the first
// remaining lambda interval is rerun once and its failing boxes are printed in
// the reference's format (e.g. middle_configuration.cu:181-183,
// end_configuration.cu:124); a second SIGINT ends the process as the reference's
// handler does.  The reference prints every failing box; the environment
// variable CP_CRITICALS_MAX (default 1048576) bounds the lines printed here.
#include <csignal>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cp_prover.h"

namespace {

const double kLambdaMin = 0.5, kLambdaMax = 0.9900000000000001;  // values.hpp:31-32

volatile std::sig_atomic_t g_interrupts = 0;
cp_prover* volatile g_active = nullptr;
void (*g_previous)(int) = SIG_DFL;

void on_sigint(int) {
    if (g_interrupts++) {
        std::signal(SIGINT, g_previous);
        std::raise(SIGINT);
        std::abort();
    }
    if (g_active) cp_request_interrupt(g_active);
}

// The reference installs its handler when a family's lambda loop starts
// (run_kernel.cuh:51-54, after the banner) and checks the flag after every
// launch.  Here the handler is installed just before the banner, and a signal
// that came before the loop started is handed to it before the first launch
// (on_step), so it takes effect after that launch as in the reference.
void arm() {
    g_interrupts = 0;
    g_previous = std::signal(SIGINT, on_sigint);
}
void disarm() { std::signal(SIGINT, g_previous); }

cp_prover* handle() {
    static cp_prover* h = nullptr;
    if (!h) {
        cp_status s = cp_create(0, &h);
        if (s != CP_OK) throw std::runtime_error(std::string("cp_create: ") + cp_status_string(s));
    }
    return h;
}

// The label of the reference's critical-interval lines, per family and handle,
// and the separator before "la = ": ": " in start_configuration.cu:147,158,207 and
// middle_configuration.cu:182,193; " - " in start_configuration.cu:289 and
// end_configuration.cu:124,135,245,256.
const char* label(int family, int handle_bit) {
    switch (family) {
    case CP_START: return handle_bit == 0 ? "Critical interval: Start configuration, case 1" : "Critical interval: Start configuration, case 2";
    case CP_START_END_2D: return "Critical interval: Start & end configuration, 2 disks";
    case CP_START_END_3D: return "Start & end configuration: Critical interval";
    case CP_MIDDLE: return handle_bit == 0 ? "Critical interval: Middle configuration, case 1.1" : "Critical interval: Middle configuration, case 2.1";
    case CP_END_2D: return handle_bit == 0 ? "End configuration (2 disks): Critical interval with r1 on the inside" : "End configuration (2 disks): Critical interval with r1 on the outside";
    default: return handle_bit == 0 ? "End configuration (3 disks): Critical interval with r1 on the inside" : "End configuration (3 disks): Critical interval with r1 on the outside";
    }
}
const char* separator(int family) {
    return (family == CP_START_END_3D || family == CP_END_2D || family == CP_END_3D) ? " - " : ": ";
}

size_t criticals_max() {
    const char* e = std::getenv("CP_CRITICALS_MAX");
    if (!e || !*e) return size_t(1) << 20;
    char* end = nullptr;
    const unsigned long long v = std::strtoull(e, &end, 10);
    return (end && *end == '\0') ? (size_t)v : (size_t(1) << 20);
}

void print_criticals(cp_prover* p, int family, double lb, double ub) {
    const size_t cap = criticals_max();
    std::vector<double> boxes(8 * (cap ? cap : 1));
    std::vector<uint8_t> handles(cap ? cap : 1);
    size_t count = 0;
    if (cp_reference_criticals(p, family, lb, ub, nullptr, cap, boxes.data(), handles.data(), &count) != CP_OK) return;
    const int dims = cp_family_dims(family);
    const char* sep = separator(family);
    for (size_t i = 0; i < count && i < cap; ++i) {
        const double* b = &boxes[8 * i];
        for (int h = 0; h < 2; ++h) {
            if (!((handles[i] >> h) & 1)) continue;
            if (dims == 4)
                std::printf("%s%sla = [%.19g,%.19g], r1 = [%.19g,%.19g], r2 = [%.19g,%.19g], r3 = [%.19g,%.19g]\n",
                            label(family, h), sep, b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7]);
            else
                std::printf("%s%sla = [%.19g,%.19g], r1 = [%.19g,%.19g], r2 = [%.19g,%.19g]\n", label(family, h), sep,
                            b[0], b[1], b[2], b[3], b[4], b[5]);
        }
    }
    std::fflush(stdout);
}

// "Handling lambda interval " followed by the interval as the reference's
// operator<< writes it (interval.hpp:295-303): right-aligned fields of width 26,
// 19 significant digits.
void on_step(void*, double lb, double ub) {
    if (g_interrupts && g_active) cp_request_interrupt(g_active);
    const std::ios_base::fmtflags flags = std::cerr.flags(std::ios::right);
    const std::streamsize prec = std::cerr.precision(19);
    std::cerr << "Handling lambda interval " << '[' << std::setw(26) << lb << ", " << std::setw(26) << ub << ']'
              << std::endl;
    std::cerr.flags(flags);
    std::cerr.precision(prec);
}

// run_kernel_until_no_criticals for one family; true when the lambda queue emptied
bool run_family(int family) {
    cp_prover* p = handle();
    g_active = p;
    cp_set_step_callback(p, on_step, nullptr);
    cp_reference_report r;
    const cp_status s = cp_prove_family_reference(p, family, kLambdaMin, kLambdaMax, nullptr, 0, nullptr, &r);
    cp_set_step_callback(p, nullptr, nullptr);
    g_active = nullptr;
    if (s == CP_ERR_INTERRUPTED) {
        std::cerr << "We were interrupted - running the first remaining interval with output once!" << std::endl;
        print_criticals(p, family, r.remaining[0], r.remaining[1]);
        return false;
    }
    if (s != CP_OK) {
        std::cerr << "lambda loop stopped: " << cp_status_string(s) << " at lambda interval [" << r.remaining[0] << ", "
                  << r.remaining[1] << "] " << cp_last_error_string() << std::endl;
        return false;
    }
    std::cerr << "lambda intervals handled: " << r.launches << ", boxes evaluated: " << r.boxes_evaluated << std::endl;
    return r.proved != 0;
}

}  // namespace

namespace circlepacking {
namespace lane_packing {

void find_critical_intervals_start_configuration() {
    arm();
    std::cout << "Start configuration..." << std::endl;
    run_family(CP_START);
    disarm();
}

void find_critical_intervals_start_end_configuration() {
    arm();
    std::cout << "Start & end configuration, 2 disks... " << std::endl;
    run_family(CP_START_END_2D);
    disarm();
    arm();
    std::cerr << "Start & end configuration, 3 disks ..." << std::endl;
    run_family(CP_START_END_3D);
    disarm();
}

void find_critical_intervals_middle_configuration() {
    arm();
    std::cout << "Middle configuration ..." << std::endl;
    run_family(CP_MIDDLE);
    disarm();
}

void find_critical_intervals_end_configuration() {
    arm();
    std::cout << "End configuration (2 disks) ..." << std::endl;
    run_family(CP_END_2D);
    disarm();
    arm();
    std::cout << "End configuration (3 disks) ..." << std::endl;
    run_family(CP_END_3D);
    disarm();
}

void find_critical_intervals() {
    find_critical_intervals_start_configuration();
    find_critical_intervals_start_end_configuration();
    find_critical_intervals_middle_configuration();
    find_critical_intervals_end_configuration();
}

}  // namespace lane_packing
}  // namespace circlepacking

// prover.cpp:33 sets the device printf FIFO; the kernels here do not print.
namespace algcuda {
namespace device {
void set_printf_buffer_size(std::size_t) {}
}  // namespace device
}  // namespace algcuda
