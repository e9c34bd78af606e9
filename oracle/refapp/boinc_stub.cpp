// Definitions behind boinc_stub/*.h: BOINC's standalone behaviour, nothing
// more.  Linked only into the reference app built by oracle/refapp/Makefile,
// a test oracle; the product never links it.
#include "boinc_api.h"
#include "mfile.h"

#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <sys/time.h>

static double g_fraction_done = 0.0;

void boinc_options_defaults(BOINC_OPTIONS& b) {
    std::memset(&b, 0, sizeof b);
    b.main_program = 1;
}

int boinc_init_options(BOINC_OPTIONS*) { return 0; }

int boinc_get_init_data(APP_INIT_DATA& aid) {
    std::memset(&aid, 0, sizeof aid);
    aid.gpu_device_num = -1;  // no client: the app reads --device from argv
    aid.gpu_usage = 1.0;
    std::strcpy(aid.gpu_type, "NVIDIA");
    return 0;
}

int boinc_get_init_data_p(APP_INIT_DATA* aid) { return boinc_get_init_data(*aid); }

char* boinc_msg_prefix(char* buf, int len) {
    std::snprintf(buf, static_cast<size_t>(len), "[standalone]");
    return buf;
}

int boinc_resolve_filename(const char* virtual_name, char* physical_name, int len) {
    std::snprintf(physical_name, static_cast<size_t>(len), "%s", virtual_name);
    return 0;
}

int boinc_resolve_filename_s(const char* virtual_name, std::string& physical_name) {
    physical_name = virtual_name;
    return 0;
}

FILE* boinc_fopen(const char* path, const char* mode) { return std::fopen(path, mode); }
int boinc_is_standalone(void) { return 1; }
int boinc_fraction_done(double fraction) { g_fraction_done = fraction; return 0; }
double boinc_get_fraction_done(void) { return g_fraction_done; }
int boinc_time_to_checkpoint(void) { return 0; }
int boinc_checkpoint_completed(void) { return 0; }
int boinc_rename(const char* old_name, const char* new_name) { return std::rename(old_name, new_name); }

int boinc_finish(int status) {
    std::fflush(nullptr);
    std::exit(status);
}

double dtime(void) {
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

int MFILE::open(const char* path, const char* mode) {
    f_ = std::fopen(path, mode);
    return f_ ? 0 : -1;
}

int MFILE::printf(const char* format, ...) {
    if (!f_) return -1;
    va_list ap;
    va_start(ap, format);
    int n = std::vfprintf(f_, format, ap);
    va_end(ap);
    return n;
}

int MFILE::flush(void) { return (f_ && std::fflush(f_) == 0) ? 0 : -1; }

int MFILE::close(void) {
    if (!f_) return 0;
    int r = std::fclose(f_);
    f_ = nullptr;
    return r;
}
