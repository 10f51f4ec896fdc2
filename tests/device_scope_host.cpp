// Host build of the device binding of the library's entry points
// (beta1_b200/csrc/mhd_device_scope.h) against a fake device API, so the
// bookkeeping is checked without a GPU: scope_trace() runs one scenario and
// writes the sequence of device calls it made.
#include "../beta1_b200/csrc/mhd_device_scope.h"

namespace
{
int g_current = 0;
int g_fail_set = -1; // device whose set() fails (-1: none)
int g_fail_get = 0;
int *g_log = nullptr;
int g_nlog = 0;

struct FakeApi
{
    static int get(int *d)
    {
        g_log[g_nlog++] = 1000;
        if (g_fail_get)
            return 1;
        *d = g_current;
        return 0;
    }
    static int set(int d)
    {
        g_log[g_nlog++] = d;
        if (d == g_fail_set)
            return 1;
        g_current = d;
        return 0;
    }
};
} // namespace

// scenario: the caller's device is `current`, the context lives on `want`
// (nested: an entry point calling another one on the same context).
// log receives 1000 for every get() and the device of every set(); returns
// ok() of the scopes * 10 + the device current after the scope ends, and
// *during the device current inside the scope.
extern "C" int scope_trace(int current, int want, int nested, int fail_set, int fail_get, int *log, int *nlog,
                           int *during)
{
    g_current = current;
    g_fail_set = fail_set;
    g_fail_get = fail_get;
    g_log = log;
    g_nlog = 0;
    int ok = 0;
    {
        DeviceScope<FakeApi> s(want);
        ok = s.ok() ? 1 : 0;
        if (nested)
        {
            DeviceScope<FakeApi> inner(want);
            ok = ok && inner.ok();
        }
        *during = g_current;
    }
    *nlog = g_nlog;
    return ok * 10 + g_current;
}
