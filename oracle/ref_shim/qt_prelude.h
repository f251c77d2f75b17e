/*
 * Minimal stand-ins for the few Qt names that CTL's matrix code uses
 * (qWarning, qFuzzyIsNull, Q_ASSERT, Qt::Axis), so that the reference's own
 * modules/src/mat/matrix_algorithm.cpp and projectionmatrix.cpp compile here
 * without Qt.  Test infrastructure for the oracle only.
 */
#ifndef CTLB200_REF_QT_PRELUDE_H
#define CTLB200_REF_QT_PRELUDE_H

#include <cassert>
#include <cmath>

struct RefShimDebugStream {
    template <typename T>
    RefShimDebugStream& operator<<(const T&) { return *this; }
};
inline RefShimDebugStream qWarning() { return RefShimDebugStream(); }
inline RefShimDebugStream qDebug() { return RefShimDebugStream(); }

/* Qt 5: qFuzzyIsNull(double d) is |d| <= 1e-12 */
inline bool qFuzzyIsNull(double d) { return std::fabs(d) <= 0.000000000001; }

#define Q_ASSERT(cond) assert(cond)

namespace Qt {
enum Axis { XAxis, YAxis, ZAxis };
}

#endif
