/* oracle/shim/table.h -- TEST INFRASTRUCTURE: the SDDS table helpers the reference
 * includes (cathode.c:16, antenna.c:16) are declared in mdb.h. */
#include "mdb.h"
