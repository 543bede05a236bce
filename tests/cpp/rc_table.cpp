// Checks of the recurrence-coefficient table layout (pfsoftlib_b200/csrc/dwt.cuh): rc_offset's
// closed form equals the running sum of B - M entries over the classes in class_orders' order,
// and rc_entries is the total. Prints "ok" and exits 0 when every check holds.
#include <math.h>

#include <cstdio>

#include "common.cuh"
#include "dwt.cuh"

int main()
{
    int failures = 0;
    for (int B = 1; B <= 512; B += (B < 40 ? 1 : 37)) {
        long long run = 0;
        for (int c = 0; c < pfsoft_dev::num_classes(B); ++c) {
            int M, Mp;
            pfsoft_dev::class_orders(c, M, Mp);
            if (pfsoft_dev::rc_offset(B, M, Mp) != run) {
                std::fprintf(stderr, "B=%d class %d (%d,%d): offset %lld, expected %lld\n", B, c, M, Mp,
                             pfsoft_dev::rc_offset(B, M, Mp), run);
                ++failures;
                break;
            }
            run += B - M;
        }
        if (pfsoft_dev::rc_entries(B) != run) {
            std::fprintf(stderr, "B=%d: %lld entries, expected %lld\n", B, pfsoft_dev::rc_entries(B), run);
            ++failures;
        }
    }
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
