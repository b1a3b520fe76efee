// Point2D.h -- small value types of the host API (IPPI-LBM/Point2D.h).
#ifndef POINT2D_H
#define POINT2D_H
#include "Parameter.h"

struct Point2D {
    REAL x;
    REAL y;
};

struct Position2D {
    int x;
    int y;
};

struct Force {
    REAL x;
    REAL y;
};

#endif
