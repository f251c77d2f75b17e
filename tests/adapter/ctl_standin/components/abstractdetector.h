// Stand-in for CTL's components/abstractdetector.h.  Test code only.
#include "../ctl_standin_types.h"
