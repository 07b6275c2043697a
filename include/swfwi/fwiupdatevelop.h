/* FwiUpdateVelOp (src/fwi/fwiupdatevelop.h:13-24); declared beside
 * UpdateVelOp. */
#include "updatevelop.h"
