/*
 * Minimal Win32 surface for compiling the reference CPU tracker on Linux.
 *
 * TEST INFRASTRUCTURE ONLY. This header is put first on the include path when
 * oracle/build_ref.py compiles a copy of the reference's cputrack/ sources into
 * oracle/_ref/libqtrk_ref.so. It maps the handful of Win32 calls those sources use
 * (threads.h: CreateMutex/WaitForSingleObject/ReleaseMutex/CreateThread/Sleep/
 * GetSystemInfo/SetThreadPriority; utils.cpp: QueryPerformanceCounter,
 * GetModuleHandleExA, GetModuleFileNameA, OutputDebugString) onto pthreads and
 * clock_gettime. Nothing in the product library includes it.
 */
#pragma once
#include <pthread.h>
#include <unistd.h>
#include <time.h>
#include <alloca.h>
#include <cstdio>
#include <cstdint>
#include <cstring>

typedef unsigned long DWORD;
typedef int BOOL;
typedef void *HANDLE;
typedef void *HMODULE;
typedef const char *LPCSTR;

#define WINAPI
#define FALSE 0
#define TRUE 1
#define INFINITE 0xffffffffUL
#define GET_MODULE_HANDLE_EX_FLAG_FROM_ADDRESS 0
#define GET_MODULE_HANDLE_EX_FLAG_UNCHANGED_REFCOUNT 0
#define THREAD_MODE_BACKGROUND_BEGIN 0
#define THREAD_MODE_BACKGROUND_END 0
#define THREAD_PRIORITY_BELOW_NORMAL 0
#define THREAD_PRIORITY_NORMAL 0

typedef union {
    long long QuadPart;
} LARGE_INTEGER;

struct OSVERSIONINFO {
    DWORD dwMajorVersion;
};
struct SYSTEM_INFO {
    DWORD dwNumberOfProcessors;
};

typedef DWORD (*LPTHREAD_START_ROUTINE)(void *);

/* One object type stands for both mutexes and threads. */
struct oracle_win_object {
    int is_thread;
    pthread_mutex_t mutex;
    pthread_t thread;
    LPTHREAD_START_ROUTINE entry;
    void *arg;
};

static inline void *oracle_thread_trampoline(void *p)
{
    oracle_win_object *o = (oracle_win_object *)p;
    o->entry(o->arg);
    return 0;
}

static inline HANDLE CreateMutex(void *, BOOL, void *)
{
    oracle_win_object *o = new oracle_win_object();
    o->is_thread = 0;
    pthread_mutexattr_t attr;
    pthread_mutexattr_init(&attr);
    /* Win32 mutexes are recursive for the owning thread. */
    pthread_mutexattr_settype(&attr, PTHREAD_MUTEX_RECURSIVE);
    pthread_mutex_init(&o->mutex, &attr);
    pthread_mutexattr_destroy(&attr);
    return o;
}

static inline HANDLE CreateThread(void *, size_t, LPTHREAD_START_ROUTINE entry, void *arg, DWORD, DWORD *id)
{
    oracle_win_object *o = new oracle_win_object();
    o->is_thread = 1;
    o->entry = entry;
    o->arg = arg;
    if (pthread_create(&o->thread, 0, oracle_thread_trampoline, o) != 0) {
        delete o;
        return 0;
    }
    if (id) *id = 0;
    return o;
}

static inline DWORD WaitForSingleObject(HANDLE h, DWORD)
{
    oracle_win_object *o = (oracle_win_object *)h;
    if (o->is_thread)
        pthread_join(o->thread, 0);
    else
        pthread_mutex_lock(&o->mutex);
    return 0;
}

static inline BOOL ReleaseMutex(HANDLE h)
{
    pthread_mutex_unlock(&((oracle_win_object *)h)->mutex);
    return TRUE;
}

static inline BOOL CloseHandle(HANDLE h)
{
    oracle_win_object *o = (oracle_win_object *)h;
    if (o && !o->is_thread) {
        pthread_mutex_destroy(&o->mutex);
        delete o;
    }
    /* thread objects are leaked on purpose: the reference joins before closing */
    return TRUE;
}

static inline void Sleep(DWORD ms) { usleep((useconds_t)ms * 1000u); }

static inline void GetSystemInfo(SYSTEM_INFO *s)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    const char *env = getenv("QTRK_REF_THREADS");
    if (env && atoi(env) > 0) n = atoi(env);
    s->dwNumberOfProcessors = (DWORD)(n > 0 ? n : 1);
}

static inline BOOL GetVersionEx(OSVERSIONINFO *v)
{
    v->dwMajorVersion = 6;
    return TRUE;
}

static inline BOOL SetThreadPriority(HANDLE, int) { return TRUE; }

static inline void OutputDebugString(const char *) {}

static inline BOOL QueryPerformanceCounter(LARGE_INTEGER *t)
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    t->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return TRUE;
}

static inline BOOL QueryPerformanceFrequency(LARGE_INTEGER *f)
{
    f->QuadPart = 1000000000LL;
    return TRUE;
}

static inline BOOL GetModuleHandleExA(DWORD, LPCSTR, HMODULE *m)
{
    if (m) *m = 0;
    return TRUE;
}

/* The reference appends its debug log next to the module: keep it in /tmp. */
static inline DWORD GetModuleFileNameA(HMODULE, char *path, DWORD n)
{
    snprintf(path, n, "/tmp/qtrk_ref_oracle.so");
    return (DWORD)strlen(path);
}
