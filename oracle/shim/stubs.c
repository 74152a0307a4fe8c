/* oracle/shim/stubs.c -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * No-op stand-ins for reference functions that perform_integration()
 * (integrate.c:149-193) calls every step but that lie outside the checked
 * path: resistors (beam snapshots, field output, field saving and
 * sampling, surface emitters and the moving window are the reference's own
 * files).  Each is inert when its
 * command was never given, which is how the checked configurations run; the
 * ones that would act bomb instead, so a checker can never silently skip
 * work.  compose_filename() stands in for the one in spiffe.c, which is not
 * compiled.
 */
#include "spiffe.h"

char *compose_filename(char *template, char *root_name)
{
  char *ptr;
  if (template && root_name && str_in(template, "%s")) {
    ptr = tmalloc(sizeof(char) * (strlen(template) + strlen(root_name) + 1));
    replace_string(ptr, template, "%s", root_name);
    return ptr;
  }
  return template;
}

void add_resistor_currents(FIELDS *EM_problem, RESISTOR *resistor)
{
  (void)EM_problem;
  (void)resistor;
  bomb("resistors are not part of the checked path", NULL);
}
