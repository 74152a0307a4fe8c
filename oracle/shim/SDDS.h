/* oracle/shim/SDDS.h -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * Project-written stand-in for the SDDS file library header, which the
 * reference includes (spiffe.h:8) but which is not in the reference tree.
 * Output datasets are captured in memory (column values per page) so a checker
 * can read back what the reference wrote, e.g. screen crossings written by
 * advance_particles.c:538-569.  Input datasets read the SDDS1 ASCII layout
 * ("&column name=... &end" lines, "&data mode=ascii", whitespace rows), which
 * is the form of the reference's example waveform file.
 */
#ifndef SPIFFE_SHIM_SDDS_H
#define SPIFFE_SHIM_SDDS_H

#include <stdio.h>
#include <stdint.h>

#define SDDS_BINARY 1
#define SDDS_ASCII 2

#define SDDS_DOUBLE 1
#define SDDS_FLOAT 2
#define SDDS_LONG 3
#define SDDS_SHORT 4
#define SDDS_STRING 5
#define SDDS_LONG64 6
#define SDDS_CHARACTER 7
#define SDDS_ANY_FLOATING_TYPE 100

#define SDDS_SET_BY_INDEX 1
#define SDDS_SET_BY_NAME 2
#define SDDS_PASS_BY_VALUE 4
#define SDDS_BY_INDEX SDDS_SET_BY_INDEX
#define SDDS_PASS_BY_REFERENCE 8

#define SDDS_EXIT_PrintErrors 1
#define SDDS_VERBOSE_PrintErrors 2
#define FLUSH_TABLE 1

#define SDDS_CHECK_OK 0
#define SDDS_CHECK_OKAY 0
#define SDDS_CHECK_NONEXISTENT 1

#define SHIM_SDDS_MAX_COLUMNS 64

typedef struct {
  int n_columns;
  char *column_name[SHIM_SDDS_MAX_COLUMNS];
  int column_type[SHIM_SDDS_MAX_COLUMNS];
  /* captured or loaded rows: one growable double array per column */
  int64_t n_rows, max_rows;
  double *data[SHIM_SDDS_MAX_COLUMNS];
  int64_t pages, page_len;
  int is_input, page_read;
} SDDS_DATASET;
typedef SDDS_DATASET SDDS_TABLE;

#define SHIM_MAX_CLOSED_TABLES 16
extern SDDS_DATASET shim_closed_tables[SHIM_MAX_CLOSED_TABLES];
extern int shim_n_closed_tables;
extern SDDS_DATASET shim_updated_tables[SHIM_MAX_CLOSED_TABLES];
extern int shim_n_updated_tables;

int32_t SDDS_InitializeOutput(SDDS_DATASET *t, int32_t data_mode, int32_t lines_per_row,
                              const char *description, const char *contents, const char *filename);
int32_t SDDS_DefineSimpleColumn(SDDS_DATASET *t, const char *name, const char *unit, int32_t type);
int32_t SDDS_DefineSimpleColumns(SDDS_DATASET *t, int32_t number, char **name, char **unit, int32_t type);
int32_t SDDS_DefineColumn(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                          const char *description, const char *format_string, int32_t type, int32_t field_length);
int32_t SDDS_DefineParameter(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                             const char *description, const char *format_string, int32_t type, char *fixed_value);
int32_t SDDS_DefineParameter1(SDDS_DATASET *t, const char *name, const char *symbol, const char *units,
                              const char *description, const char *format_string, int32_t type, void *fixed_value);
int32_t SDDS_WriteLayout(SDDS_DATASET *t);
int32_t SDDS_SaveLayout(SDDS_DATASET *t);
int32_t SDDS_StartPage(SDDS_DATASET *t, int64_t expected_n_rows);
int32_t SDDS_StartTable(SDDS_DATASET *t, int64_t expected_n_rows);
int32_t SDDS_SetRowValues(SDDS_DATASET *t, int32_t mode, int64_t row, ...);
int32_t SDDS_GetColumnIndex(SDDS_DATASET *t, char *name);
int32_t SDDS_NumberOfErrors(void);
int32_t SDDS_SetColumn(SDDS_DATASET *t, int32_t mode, void *data, int64_t rows, ...);
int32_t SDDS_SetParameters(SDDS_DATASET *t, int32_t mode, ...);
int32_t SDDS_WritePage(SDDS_DATASET *t);
int32_t SDDS_WriteTable(SDDS_DATASET *t);
int32_t SDDS_UpdatePage(SDDS_DATASET *t, uint32_t mode);
#define SDDS_UpdateTable(t) SDDS_UpdatePage(t, 0)
int32_t SDDS_Terminate(SDDS_DATASET *t);
void SDDS_SetError(char *error_text);
void SDDS_PrintErrors(FILE *fp, int32_t mode);
void SDDS_Bomb(char *message);
void *SDDS_Realloc(void *old_ptr, size_t new_size);
int32_t SDDS_CopyString(char **target, const char *source);
int32_t SDDS_ZeroMemory(void *mem, int64_t n_bytes);
int32_t SDDS_CheckTableStructureSize(size_t size);
int32_t SDDS_InitializeInput(SDDS_DATASET *t, char *filename);
int32_t SDDS_ReadPage(SDDS_DATASET *t);
int64_t SDDS_CountRowsOfInterest(SDDS_DATASET *t);
int64_t SDDS_RowCount(SDDS_DATASET *t);
double *SDDS_GetColumnInDoubles(SDDS_DATASET *t, char *column_name);
int32_t SDDS_CheckColumn(SDDS_DATASET *t, char *name, char *units, int32_t type, FILE *fp_message);

/* checker helpers (not part of SDDS): rows captured for one column */
int64_t shim_sdds_column(SDDS_DATASET *t, const char *name, double **values);

#endif
