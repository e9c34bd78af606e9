// Minimal stand-in for the BOINC client API, written for this project so the
// reference's unmodified GPU app (period_search_BOINC.cpp, start_CUDA.cu) can
// be built and run standalone as a test oracle and speed bar.  Only the names
// the app uses exist here; each behaves as BOINC does for a standalone run
// (no client attached): file names resolve to themselves, checkpoints are
// always due, progress reports are dropped, and boinc_finish() exits.
// Test infrastructure only: nothing in the product links this.
#pragma once
#include <cstdio>
#include <string>

struct BOINC_OPTIONS {
    int main_program;
    int check_heartbeat;
    int handle_process_control;
    int send_status_msgs;
    int direct_process_action;
    int multi_thread;
    int multi_process;
    int normal_thread_priority;
};

struct APP_INIT_DATA {
    int major_version;
    int minor_version;
    int release;
    int app_version;
    int slot;
    int gpu_device_num;
    double gpu_usage;
    char gpu_type[64];
};

void boinc_options_defaults(BOINC_OPTIONS& b);
int boinc_init_options(BOINC_OPTIONS* opt);
int boinc_get_init_data(APP_INIT_DATA& aid);
int boinc_get_init_data_p(APP_INIT_DATA* aid);
char* boinc_msg_prefix(char* buf, int len);
int boinc_resolve_filename(const char* virtual_name, char* physical_name, int len);
int boinc_resolve_filename_s(const char* virtual_name, std::string& physical_name);
FILE* boinc_fopen(const char* path, const char* mode);
int boinc_is_standalone(void);
int boinc_fraction_done(double fraction);
double boinc_get_fraction_done(void);
int boinc_time_to_checkpoint(void);
int boinc_checkpoint_completed(void);
int boinc_rename(const char* old_name, const char* new_name);
int boinc_finish(int status);
double dtime(void);
