// Upstream argument rules shared by the entry points: HOWMNY decoding, the selection count
// (a complex pair counts when either of its flags is set) and INFO = -2 / -16
// (src/dtgevc3.cpp:1172-1216, src/ztgevc3.cpp:457-490).
#pragma once

namespace xtg {

// Returns true when the caller should stop (info set, *m reported).  `count` receives the
// number of eigenvector columns.
template <class R>
bool check_args(bool cplx, char howmny, const int *select, int n, const R *alphai, int mm, int *m, int *info,
                int *count)
{
    const bool do_all = howmny == 'A' || howmny == 'B';
    const bool do_sel = howmny == 'S';
    if (!do_all && !do_sel) {
        *info = -2;
        return true;
    }
    if (n == 0) {
        *info = 0;
        if (m) *m = 0;
        return true;
    }
    int num = 0;
    for (int k = 0; k < n;) {
        const bool pair = !cplx && alphai[k] != R(0) && k + 1 < n;
        bool sel = do_all;
        if (do_sel) sel = select && (select[k] != 0 || (pair && select[k + 1] != 0));
        if (sel) num += pair ? 2 : 1;
        k += pair ? 2 : 1;
    }
    if (m) *m = num;
    if (mm < num) {
        *info = -16;
        return true;
    }
    *count = num;
    return false;
}

}  // namespace xtg
