/* FwiUpdateSteplenOp (src/fwi/fwiupdatesteplenop.h:15-45); declared beside
 * UpdateSteplenOp. */
#include "updatesteplenop.h"
