#include "qt_prelude.h"
