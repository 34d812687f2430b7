// CPU check of gb::host::SymbolAddressCache (geobrain_b200/csrc/gb_symcache.h),
// the per-(device, context) cache of the static scratch array's address that
// gb_forward_static_scratch uses.  Prints "ok" and exits 0 when every check
// holds.
#include "../geobrain_b200/csrc/gb_symcache.h"

#include <cstdio>

static int failures = 0;
#define CHECK(cond)                                                      \
    do {                                                                 \
        if (!(cond)) {                                                   \
            std::printf("check failed at line %d: %s\n", __LINE__, #cond); \
            ++failures;                                                  \
        }                                                                \
    } while (0)

int main()
{
    gb::host::SymbolAddressCache<4> cache;
    char module_a[1], module_b[1], module_c[1];
    void *next = module_a;     // the address the next lookup reports
    int calls = 0;
    auto lookup = [&](void **addr) {
        ++calls;
        *addr = next;
        return 0;
    };
    void *p = nullptr;
    // first call on device 0, context 7: one lookup
    CHECK(cache.get(0, 7, lookup, &p) == 0 && p == module_a && calls == 1);
    // same device and context: cached, no lookup even if the module moved
    next = module_b;
    CHECK(cache.get(0, 7, lookup, &p) == 0 && p == module_a && calls == 1);
    // same device, a new context (after a reset, or a host's own context): fresh lookup
    CHECK(cache.get(0, 8, lookup, &p) == 0 && p == module_b && calls == 2);
    // the first context keeps its own address
    CHECK(cache.get(0, 7, lookup, &p) == 0 && p == module_a && calls == 2);
    // another device with the same context number is another key
    next = module_c;
    CHECK(cache.get(1, 8, lookup, &p) == 0 && p == module_c && calls == 3);
    // a failed lookup returns its code and caches nothing
    auto failing = [&](void **) { ++calls; return -2; };
    CHECK(cache.get(2, 9, failing, &p) == -2 && calls == 4);
    CHECK(cache.get(2, 9, lookup, &p) == 0 && p == module_c && calls == 5);
    // a full table drops its oldest entry, which is then looked up again
    CHECK(cache.get(3, 10, lookup, &p) == 0 && calls == 6);        // entries: (0,7) (0,8) (1,8) (2,9) -> full
    next = module_b;
    CHECK(cache.get(0, 7, lookup, &p) == 0 && p == module_b && calls == 7);
    CHECK(cache.lookups() == 6);
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
