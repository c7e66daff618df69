/* TEST INFRASTRUCTURE ONLY. (Every model of the oracle is restated; this
 * translation unit is kept empty so the build's source list stays stable.) */
#include "cep_oracle.h"
