/* oracle/shim/shim.c -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * Implementations behind the project-written stand-ins for the SDDS toolkit
 * headers (mdb.h, namelist.h, SDDS.h) that the reference spiffe sources need
 * in order to compile in place.  Nothing here is reference code; where the
 * SDDS library defines an algorithm (random numbers, table interpolation,
 * elliptic integrals) this file uses the project's own published-method
 * version, and the CUDA path uses the same one, so both sides agree.
 */
#include <ctype.h>
#include <stdarg.h>
#include "mdb.h"
#include "namelist.h"
#include "SDDS.h"

/* ------------------------------------------------------------------ errors */

void bomb(char *error, char *usage)
{
  if (error)
    fprintf(stderr, "error: %s\n", error);
  if (usage)
    fprintf(stderr, "usage: %s\n", usage);
  exit(1);
}

/* -------------------------------------------------------------- allocation */

void *tmalloc(uint64_t size)
{
  void *p = calloc(1, size ? size : 1);
  if (!p)
    bomb("allocation failure in tmalloc", NULL);
  return p;
}

void *trealloc(void *ptr, uint64_t size)
{
  void *p = realloc(ptr, size ? size : 1);
  if (!p)
    bomb("allocation failure in trealloc", NULL);
  return p;
}

void *array_1d(uint64_t size_of_elem, int64_t lower, int64_t upper)
{
  char *p = tmalloc(size_of_elem * (uint64_t)(upper - lower + 1));
  return p - size_of_elem * lower;
}

/* Row-pointer 2-D array over one zeroed contiguous block, so a checker can
 * hand the reference a contiguous buffer it owns. */
void **zarray_2d(uint64_t size, uint64_t n1, uint64_t n2)
{
  char *block = tmalloc(size * n1 * n2);
  void **rows = tmalloc(sizeof(void *) * n1);
  uint64_t i;
  for (i = 0; i < n1; i++)
    rows[i] = block + size * n2 * i;
  return rows;
}

int free_zarray_2d(void **array, uint64_t n1, uint64_t n2)
{
  (void)n1;
  (void)n2;
  if (array) {
    free(array[0]);
    free(array);
  }
  return 1;
}

/* --------------------------------------------------------------------- RNG
 * Counter-based generator: the k-th draw of stream `key` is the SplitMix64
 * finaliser (Steele, Lea & Flood, OOPSLA 2014; constants of Stafford's
 * "variant 13") applied to key + (k+1)*golden, keeping the top 53 bits.  The
 * product computes the same function on the host and on the device. */
static uint64_t rng_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static uint64_t rng_key = 0, rng_counter = 0;

double random_1(long iseed)
{
  if (iseed < 0) {
    rng_key = rng_mix64((uint64_t)(-iseed) * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL);
    rng_counter = 0;
    return 0.0;
  }
  rng_counter++;
  return (double)(rng_mix64(rng_key + rng_counter * 0x9E3779B97F4A7C15ULL) >> 11) * 0x1.0p-53;
}

/* random_2, the second stream (the surface emitters', emitter.c:63, :276,
 * :306, :328): the same generator under another key derivation */
static uint64_t rng2_key = 0, rng2_counter = 0;

double random_2(long iseed)
{
  if (iseed < 0) {
    rng2_key = rng_mix64((uint64_t)(-iseed) * 0x9E3779B97F4A7C15ULL + 0xD1B54A32D192ED03ULL);
    rng2_counter = 0;
    return 0.0;
  }
  rng2_counter++;
  return (double)(rng_mix64(rng2_key + rng2_counter * 0x9E3779B97F4A7C15ULL) >> 11) * 0x1.0p-53;
}

/* checker hook: position of the shared stream */
uint64_t shim_rng_counter(void) { return rng_counter; }

double gauss_rn_lim(double mean, double sigma, double limit_in_sigmas, double (*urandom)(long iseed))
{
  /* Box-Muller; redraw while outside the limit when a limit is given */
  double u1, u2, x;
  do {
    do
      u1 = urandom(1);
    while (u1 <= 0);
    u2 = urandom(1);
    x = sqrt(-2 * log(u1)) * cos(PIx2 * u2);
  } while (limit_in_sigmas > 0 && fabs(x) > limit_in_sigmas);
  return mean + sigma * x;
}

#define MAX_HALTON 16
static int32_t halton_radix[MAX_HALTON];
static int64_t halton_index[MAX_HALTON];
static int32_t n_halton = 0;

int32_t startHaltonSequence(int32_t *radix, double value)
{
  (void)value;
  if (n_halton >= MAX_HALTON)
    bomb("too many Halton sequences", NULL);
  halton_radix[n_halton] = *radix;
  halton_index[n_halton] = 0;
  return n_halton++;
}

double nextHaltonSequencePoint(long ID)
{
  /* radical inverse of the running index in the sequence's radix */
  int64_t i = ++halton_index[ID];
  double f = 1, r = 0;
  while (i > 0) {
    f /= halton_radix[ID];
    r += f * (i % halton_radix[ID]);
    i /= halton_radix[ID];
  }
  return r;
}

/* -------------------------------------------------------------- numerics */

/* Linear interpolation in an ascending table; outside it returns the end
 * value and sets *returnCode to 0. */
double interp(double *f, double *x, long n, double xo, long warnings, long order, long *returnCode)
{
  long lo, hi, mid;
  (void)warnings;
  (void)order;
  *returnCode = 1;
  if (n < 1)
    return 0;
  if (xo <= x[0]) {
    if (xo < x[0])
      *returnCode = 0;
    return f[0];
  }
  if (xo >= x[n - 1]) {
    if (xo > x[n - 1])
      *returnCode = 0;
    return f[n - 1];
  }
  lo = 0;
  hi = n - 1;
  while (hi - lo > 1) {
    mid = (lo + hi) / 2;
    if (x[mid] <= xo)
      lo = mid;
    else
      hi = mid;
  }
  return f[lo] + (f[hi] - f[lo]) / (x[hi] - x[lo]) * (xo - x[lo]);
}

/* Complete elliptic integrals of the first and second kind of modulus k by
 * the arithmetic-geometric mean (Abramowitz & Stegun 17.6).  The product's
 * solenoid setup evaluates the same iteration. */
static void agm_cei(double k, double *K, double *E)
{
  double a = 1, b = sqrt(1 - k * k), c = k, sum = 0.5 * k * k, pow2 = 0.5, an;
  int n;
  for (n = 0; n < 60 && fabs(c) > 1e-17; n++) {
    an = (a + b) / 2;
    c = (a - b) / 2;
    b = sqrt(a * b);
    a = an;
    pow2 *= 2;
    sum += pow2 * c * c;
  }
  *K = PI / (2 * a);
  *E = *K * (1 - sum);
}

double K_cei(double k)
{
  double K, E;
  agm_cei(k, &K, &E);
  return K;
}

double E_cei(double k)
{
  double K, E;
  agm_cei(k, &K, &E);
  return E;
}

double ipow(double x, long p)
{
  double r = 1;
  long i;
  if (p < 0)
    return 1 / ipow(x, -p);
  for (i = 0; i < p; i++)
    r *= x;
  return r;
}

long binaryArraySearch(void *array, size_t elementSize, long elements, void *key,
                       int (*compare)(const void *c1, const void *c2), long bracket)
{
  long lo = 0, hi = elements - 1, mid;
  char *a = array;
  (void)bracket;
  if (elements <= 0 || compare(key, a) < 0)
    return -1;
  if (compare(key, a + elementSize * hi) >= 0)
    return hi;
  while (hi - lo > 1) {
    mid = (lo + hi) / 2;
    if (compare(key, a + elementSize * mid) >= 0)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

long computeMoments(double *mean, double *rms, double *standDev, double *meanAbsoluteDev, double *x, long n)
{
  long i;
  double s = 0, s2 = 0, sd = 0, mad = 0, m;
  if (n <= 0)
    return 0;
  for (i = 0; i < n; i++) {
    s += x[i];
    s2 += x[i] * x[i];
  }
  m = s / n;
  for (i = 0; i < n; i++) {
    sd += (x[i] - m) * (x[i] - m);
    mad += fabs(x[i] - m);
  }
  if (mean)
    *mean = m;
  if (rms)
    *rms = sqrt(s2 / n);
  if (standDev)
    *standDev = n > 1 ? sqrt(sd / (n - 1)) : 0;
  if (meanAbsoluteDev)
    *meanAbsoluteDev = mad / n;
  return 1;
}

int find_min_max(double *min, double *max, double *list, int64_t n)
{
  int64_t i;
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (i = 0; i < n; i++) {
    if (list[i] < lo)
      lo = list[i];
    if (list[i] > hi)
      hi = list[i];
  }
  if (min)
    *min = lo;
  if (max)
    *max = hi;
  return n > 0;
}

void SavitzkyGolaySmooth(double *data, long rows, long order, long nLeft, long nRight, long derivativeOrder)
{
  (void)data;
  (void)rows;
  (void)order;
  (void)nLeft;
  (void)nRight;
  (void)derivativeOrder;
  bomb("Savitzky-Golay current smoothing is not part of the checked path", NULL);
}

/* ----------------------------------------------------------------- strings */

long match_string(char *string, char **option, long n_options, long mode)
{
  long i, hit = -1, hits = 0, len;
  if (!string)
    return -1;
  for (i = 0; i < n_options; i++)
    if (strcmp(string, option[i]) == 0)
      return i;
  if (mode & EXACT_MATCH)
    return -1;
  len = (long)strlen(string);
  for (i = 0; i < n_options; i++)
    if (strncmp(string, option[i], len) == 0) {
      hit = i;
      hits++;
    }
  return hits == 1 ? hit : -1;
}

char *str_tolower(char *s)
{
  char *p;
  for (p = s; *p; p++)
    *p = (char)tolower((unsigned char)*p);
  return s;
}

char *str_in(char *s, char *t) { return strstr(s, t); }

char *replace_string(char *target, char *source, char *orig, char *newStr)
{
  char *hit = strstr(source, orig);
  if (!hit) {
    strcpy(target, source);
    return target;
  }
  memcpy(target, source, (size_t)(hit - source));
  strcpy(target + (hit - source), newStr);
  strcat(target, hit + strlen(orig));
  return target;
}

char *cp_str(char **s, char *t)
{
  *s = t ? strdup(t) : NULL;
  return *s;
}

FILE *fopen_e(char *file, char *open_mode, long mode)
{
  FILE *fp = fopen(file, open_mode);
  (void)mode;
  if (!fp) {
    fprintf(stderr, "unable to open %s\n", file);
    exit(1);
  }
  return fp;
}

/* --------------------------------------------------------------- namelists
 * Text form: "&group name=value, name="string" ... &end" (a lone "&" also
 * ends a group, as in the reference's example boundary files); lines whose
 * first non-blank character is '!' are comments. */

char *get_namelist(char *s, long n, FILE *fp)
{
  char line[4096];
  long used = 0;
  int started = 0;
  s[0] = 0;
  while (fgets(line, sizeof(line), fp)) {
    char *p = line, *amp;
    while (*p && isspace((unsigned char)*p))
      p++;
    if (*p == '!' || (!started && *p != '&'))
      continue;
    started = 1;
    if (used + (long)strlen(p) + 2 >= n)
      bomb("namelist too long", NULL);
    strcpy(s + used, p);
    used += (long)strlen(p);
    s[used++] = ' ';
    s[used] = 0;
    /* a group ends at "&end" or at a second '&' */
    amp = strchr(s + 1, '&');
    if (amp)
      return s;
  }
  return started ? s : NULL;
}

static char *skip_sep(char *p)
{
  while (*p && (isspace((unsigned char)*p) || *p == ','))
    p++;
  return p;
}

long scan_namelist(NAMELIST_TEXT *text, char *s)
{
  char *p = s, *q;
  long cap = 16;
  memset(text, 0, sizeof(*text));
  while (*p && *p != '&')
    p++;
  if (!*p)
    return 0;
  p++;
  q = p;
  while (*q && !isspace((unsigned char)*q) && *q != '&')
    q++;
  text->group_name = strndup(p, (size_t)(q - p));
  text->entity = malloc(sizeof(char *) * cap);
  text->value = malloc(sizeof(char *) * cap);
  p = q;
  for (;;) {
    char *name, *value;
    p = skip_sep(p);
    if (!*p || *p == '&' || *p == '$')
      break;
    q = p;
    while (*q && *q != '=' && !isspace((unsigned char)*q))
      q++;
    name = strndup(p, (size_t)(q - p));
    p = q;
    while (*p && isspace((unsigned char)*p))
      p++;
    if (*p != '=')
      bomb("namelist syntax: expected '='", NULL);
    p++;
    while (*p && isspace((unsigned char)*p))
      p++;
    if (*p == '"') {
      q = strchr(p + 1, '"');
      if (!q)
        bomb("namelist syntax: unterminated string", NULL);
      value = strndup(p + 1, (size_t)(q - p - 1));
      p = q + 1;
    } else {
      q = p;
      while (*q && *q != ',' && *q != '&' && !isspace((unsigned char)*q))
        q++;
      value = strndup(p, (size_t)(q - p));
      p = q;
    }
    if (text->n_entities == cap) {
      cap *= 2;
      text->entity = realloc(text->entity, sizeof(char *) * cap);
      text->value = realloc(text->value, sizeof(char *) * cap);
    }
    text->entity[text->n_entities] = name;
    text->value[text->n_entities] = value;
    text->n_entities++;
  }
  return 1;
}

long process_namelist(NAMELIST *nl, NAMELIST_TEXT *text)
{
  long i, j;
  for (i = 0; i < text->n_entities; i++) {
    for (j = 0; j < nl->n_items; j++)
      if (strcasecmp(text->entity[i], nl->item[j].name) == 0)
        break;
    if (j == nl->n_items) {
      fprintf(stderr, "unknown variable %s in namelist %s\n", text->entity[i], nl->group_name);
      exit(1);
    }
    switch (nl->item[j].type) {
    case NL_DOUBLE:
      *(double *)nl->item[j].address = strtod(text->value[i], NULL);
      break;
    case NL_LONG:
      *(long *)nl->item[j].address = (long)strtod(text->value[i], NULL);
      break;
    case NL_INT:
      *(int *)nl->item[j].address = (int)strtod(text->value[i], NULL);
      break;
    case NL_SHORT:
      *(short *)nl->item[j].address = (short)strtod(text->value[i], NULL);
      break;
    case NL_STRING:
      *(char **)nl->item[j].address = strdup(text->value[i]);
      break;
    }
  }
  return 0;
}

void print_namelist(FILE *fp, NAMELIST *nl)
{
  (void)fp;
  (void)nl;
}

void free_namelist_text(NAMELIST_TEXT *text)
{
  long i;
  for (i = 0; i < text->n_entities; i++) {
    free(text->entity[i]);
    free(text->value[i]);
  }
  free(text->entity);
  free(text->value);
  free(text->group_name);
  memset(text, 0, sizeof(*text));
}

/* --------------------------------------------------------------------- SDDS */

static char *shim_last_error = NULL;

static int col_index(SDDS_DATASET *t, const char *name)
{
  int i;
  for (i = 0; i < t->n_columns; i++)
    if (strcmp(t->column_name[i], name) == 0)
      return i;
  return -1;
}

/* grows every column to hold `rows`; only the new slots are cleared (rows of
 * the page being assembled, beyond n_rows, may already hold values) */
static void ensure_rows(SDDS_DATASET *t, int64_t rows)
{
  int i;
  const int64_t old = t->max_rows;
  if (rows <= t->max_rows)
    return;
  while (t->max_rows < rows)
    t->max_rows = t->max_rows ? 2 * t->max_rows : 1024;
  for (i = 0; i < t->n_columns; i++) {
    t->data[i] = trealloc(t->data[i], sizeof(double) * (uint64_t)t->max_rows);
    memset(t->data[i] + old, 0, sizeof(double) * (uint64_t)(t->max_rows - old));
  }
}

/* rows of the page being assembled start at n_rows; pages counts writes */

int32_t SDDS_InitializeOutput(SDDS_DATASET *t, int32_t data_mode, int32_t lines_per_row,
                              const char *description, const char *contents, const char *filename)
{
  (void)data_mode;
  (void)lines_per_row;
  (void)description;
  (void)contents;
  (void)filename;
  memset(t, 0, sizeof(*t));
  return 1;
}

int32_t SDDS_DefineSimpleColumn(SDDS_DATASET *t, const char *name, const char *unit, int32_t type)
{
  (void)unit;
  if (t->n_columns >= SHIM_SDDS_MAX_COLUMNS)
    return 0;
  t->column_name[t->n_columns] = strdup(name);
  t->column_type[t->n_columns] = type;
  t->data[t->n_columns] = NULL;
  t->n_columns++;
  return 1;
}

int32_t SDDS_DefineSimpleColumns(SDDS_DATASET *t, int32_t number, char **name, char **unit, int32_t type)
{
  int32_t i;
  for (i = 0; i < number; i++)
    if (!SDDS_DefineSimpleColumn(t, name[i], unit ? unit[i] : NULL, type))
      return 0;
  return 1;
}

int32_t SDDS_DefineColumn(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                          const char *description, const char *format_string, int32_t type, int32_t field_length)
{
  (void)symbol;
  (void)description;
  (void)format_string;
  (void)field_length;
  if (!SDDS_DefineSimpleColumn(t, name, units, type))
    return -1;
  return t->n_columns - 1;
}

int32_t SDDS_DefineParameter(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                             const char *description, const char *format_string, int32_t type, char *fixed_value)
{
  (void)t; (void)name; (void)symbol; (void)units; (void)description; (void)format_string; (void)type; (void)fixed_value;
  return 0;
}

int32_t SDDS_DefineParameter1(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                              const char *description, const char *format_string, int32_t type, void *fixed_value)
{
  (void)t; (void)name; (void)symbol; (void)units; (void)description; (void)format_string; (void)type; (void)fixed_value;
  return 0;
}

int32_t SDDS_WriteLayout(SDDS_DATASET *t) { (void)t; return 1; }
int32_t SDDS_SaveLayout(SDDS_DATASET *t) { (void)t; return 1; }

int32_t SDDS_StartPage(SDDS_DATASET *t, int64_t expected_n_rows)
{
  (void)t;
  (void)expected_n_rows;
  t->page_len = 0;
  return 1;
}

int32_t SDDS_StartTable(SDDS_DATASET *t, int64_t expected_n_rows) { return SDDS_StartPage(t, expected_n_rows); }

int32_t SDDS_SetRowValues(SDDS_DATASET *t, int32_t mode, int64_t row, ...)
{
  va_list ap;
  va_start(ap, row);
  ensure_rows(t, t->n_rows + row + 1);
  for (;;) {
    int c;
    double v;
    if (mode & SDDS_SET_BY_INDEX) {
      c = va_arg(ap, int32_t);
      if (c < 0)
        break;
    } else {
      char *name = va_arg(ap, char *);
      if (!name)
        break;
      c = col_index(t, name);
      if (c < 0)
        bomb("SDDS_SetRowValues: unknown column", NULL);
    }
    if (t->column_type[c] == SDDS_DOUBLE || t->column_type[c] == SDDS_FLOAT)
      v = va_arg(ap, double);
    else
      v = (double)va_arg(ap, int);
    t->data[c][t->n_rows + row] = v;
  }
  va_end(ap);
  if (row + 1 > t->page_len)
    t->page_len = row + 1;
  return 1;
}

int32_t SDDS_SetColumn(SDDS_DATASET *t, int32_t mode, void *data, int64_t rows, ...)
{
  va_list ap;
  int c;
  int64_t i;
  va_start(ap, rows);
  if (mode & SDDS_SET_BY_INDEX)
    c = va_arg(ap, int32_t);
  else
    c = col_index(t, va_arg(ap, char *));
  va_end(ap);
  if (c < 0 || c >= t->n_columns)
    bomb("SDDS_SetColumn: unknown column", NULL);
  ensure_rows(t, t->n_rows + rows);
  for (i = 0; i < rows; i++) {
    double v;
    switch (t->column_type[c]) {
    case SDDS_DOUBLE: v = ((double *)data)[i]; break;
    case SDDS_FLOAT: v = ((float *)data)[i]; break;
    case SDDS_SHORT: v = ((short *)data)[i]; break;
    default: v = ((int32_t *)data)[i]; break;
    }
    t->data[c][t->n_rows + i] = v;
  }
  if (rows > t->page_len)
    t->page_len = rows;
  return 1;
}

int32_t SDDS_SetParameters(SDDS_DATASET *t, int32_t mode, ...)
{
  (void)t;
  (void)mode;
  return 1;
}

int32_t SDDS_WritePage(SDDS_DATASET *t)
{
  t->n_rows += t->page_len;
  t->page_len = 0;
  t->pages++;
  return 1;
}

int32_t SDDS_WriteTable(SDDS_DATASET *t) { return SDDS_WritePage(t); }

int32_t SDDS_GetColumnIndex(SDDS_DATASET *t, char *name) { return col_index(t, name); }
int32_t SDDS_NumberOfErrors(void) { return 0; }
/* Tables written row by row with SDDS_UpdatePage and never closed (the
 * status file lives on perform_integration's stack, integrate.c:50, :79-80):
 * a copy of each, by its address, taken at every update; the rows stay on
 * the heap after the function returns. */
SDDS_DATASET shim_updated_tables[SHIM_MAX_CLOSED_TABLES];
static const void *shim_updated_keys[SHIM_MAX_CLOSED_TABLES];
int shim_n_updated_tables;

int32_t SDDS_UpdatePage(SDDS_DATASET *t, uint32_t mode)
{
  int k;
  (void)mode;
  /* the rows set so far stay on the open page (row numbers count from its
     start), so the page is not advanced */
  for (k = 0; k < shim_n_updated_tables; k++)
    if (shim_updated_keys[k] == t)
      break;
  if (k < SHIM_MAX_CLOSED_TABLES) {
    if (k == shim_n_updated_tables)
      shim_updated_keys[shim_n_updated_tables++] = t;
    shim_updated_tables[k] = *t;
    shim_updated_tables[k].n_rows = t->n_rows + t->page_len;
    shim_updated_tables[k].pages = t->pages + 1;
  }
  return 1;
}
/* Output tables the reference closes inside a command (a local dataset, as
 * for add_on_axis_fields' fields_used file, onAxisFields.c:130-170) are kept
 * here, in the order they were closed, so the checker can still read them. */
SDDS_DATASET shim_closed_tables[SHIM_MAX_CLOSED_TABLES];
int shim_n_closed_tables;

int32_t SDDS_Terminate(SDDS_DATASET *t)
{
  if (!t->is_input && t->n_columns && shim_n_closed_tables < SHIM_MAX_CLOSED_TABLES)
    shim_closed_tables[shim_n_closed_tables++] = *t;
  return 1;
}

void SDDS_SetError(char *error_text)
{
  free(shim_last_error);
  shim_last_error = error_text ? strdup(error_text) : NULL;
}

void SDDS_PrintErrors(FILE *fp, int32_t mode)
{
  if (shim_last_error)
    fprintf(fp, "SDDS error: %s\n", shim_last_error);
  if (mode & SDDS_EXIT_PrintErrors)
    exit(1);
}

void SDDS_Bomb(char *message) { bomb(message, NULL); }

void *SDDS_Realloc(void *old_ptr, size_t new_size) { return realloc(old_ptr, new_size ? new_size : 1); }

int32_t SDDS_CopyString(char **target, const char *source)
{
  *target = source ? strdup(source) : NULL;
  return 1;
}

int32_t SDDS_ZeroMemory(void *mem, int64_t n_bytes)
{
  memset(mem, 0, (size_t)n_bytes);
  return 1;
}

int32_t SDDS_CheckTableStructureSize(size_t size) { (void)size; return 1; }

int32_t SDDS_InitializeInput(SDDS_DATASET *t, char *filename)
{
  FILE *fp = fopen(filename, "r");
  char line[4096];
  int in_data = 0, row_counts = 1, count_seen = 0;
  memset(t, 0, sizeof(*t));
  t->is_input = 1;
  if (!fp)
    return 0;
  while (fgets(line, sizeof(line), fp)) {
    if (!in_data) {
      char *p = strstr(line, "&column");
      if (p) {
        char *n = strstr(p, "name="), *e;
        if (!n)
          continue;
        n += 5;
        e = n;
        while (*e && *e != ',' && !isspace((unsigned char)*e) && *e != '&')
          e++;
        SDDS_DefineSimpleColumn(t, strndup(n, (size_t)(e - n)), NULL, SDDS_DOUBLE);
      } else if (strstr(line, "&data")) {
        in_data = 1;
        if (strstr(line, "no_row_counts=1"))
          row_counts = 0;
      }
      continue;
    }
    {
      char *p = line, *end;
      int c;
      while (*p && isspace((unsigned char)*p))
        p++;
      if (!*p || *p == '!')
        continue;
      if (row_counts && !count_seen) {
        count_seen = 1;
        continue;
      }
      ensure_rows(t, t->n_rows + 1);
      for (c = 0; c < t->n_columns; c++) {
        t->data[c][t->n_rows] = strtod(p, &end);
        p = end;
      }
      t->n_rows++;
    }
  }
  fclose(fp);
  return 1;
}

int32_t SDDS_ReadPage(SDDS_DATASET *t)
{
  if (t->page_read)
    return -1;
  t->page_read = 1;
  return 1;
}

int64_t SDDS_CountRowsOfInterest(SDDS_DATASET *t) { return t->n_rows; }
int64_t SDDS_RowCount(SDDS_DATASET *t) { return t->n_rows; }

double *SDDS_GetColumnInDoubles(SDDS_DATASET *t, char *column_name)
{
  int c = col_index(t, column_name);
  double *v;
  if (c < 0)
    return NULL;
  v = tmalloc(sizeof(double) * (uint64_t)(t->n_rows ? t->n_rows : 1));
  memcpy(v, t->data[c], sizeof(double) * (size_t)t->n_rows);
  return v;
}

int32_t SDDS_CheckColumn(SDDS_DATASET *t, char *name, char *units, int32_t type, FILE *fp_message)
{
  (void)units;
  (void)type;
  (void)fp_message;
  return col_index(t, name) >= 0 ? SDDS_CHECK_OK : SDDS_CHECK_NONEXISTENT;
}

int64_t shim_sdds_column(SDDS_DATASET *t, const char *name, double **values)
{
  int c = col_index(t, name);
  if (c < 0) {
    *values = NULL;
    return 0;
  }
  *values = t->data[c];
  return t->n_rows;
}
