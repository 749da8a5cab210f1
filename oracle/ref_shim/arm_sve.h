// Host stand-in for <arm_sve.h>: the SVE subset lives with the SME subset.
#include "arm_sme.h"
