/* oracle/shim/namelist.h -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * Project-written stand-in for the SDDS `namelist.h` library header and the
 * tables its `nlpp` code generator writes (the reference includes generated
 * headers such as integrate.h inside its setup functions, e.g. integrate.c:47).
 * A NAMELIST is a named table of (variable name, type, address); NAMELIST_TEXT
 * holds one parsed "&group name=value, ... &end" block.  process_namelist()
 * assigns the parsed values to the variables; parsing is in oracle/shim/shim.c.
 */
#ifndef SPIFFE_SHIM_NAMELIST_H
#define SPIFFE_SHIM_NAMELIST_H

#include <stdio.h>
#include <stdint.h>

#define NL_DOUBLE 1
#define NL_LONG 2
#define NL_INT 3
#define NL_SHORT 4
#define NL_STRING 5

typedef char *STRING;

typedef struct {
  const char *name;
  int type;
  void *address;
} NL_ITEM;

typedef struct {
  NL_ITEM *item;
  const char *group_name;
  long n_items;
} NAMELIST;

typedef struct {
  char *group_name;
  long n_entities;
  char **entity;
  char **value;
} NAMELIST_TEXT;

#define NL_ENTRY(var, kind) {#var, kind, (void *)&(var)}
#define NL_DEFINE(group, items) \
  static NAMELIST group = {items, #group, (long)(sizeof(items) / sizeof(items[0]))}

long process_namelist(NAMELIST *nl, NAMELIST_TEXT *text);
void print_namelist(FILE *fp, NAMELIST *nl);
long scan_namelist(NAMELIST_TEXT *text, char *s);
char *get_namelist(char *s, long n, FILE *fp);
void free_namelist_text(NAMELIST_TEXT *text);

#endif
