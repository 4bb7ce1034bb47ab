/*
 * filter_split_sets_by_min <min_members> <prefix> <split_set...>
 *
 * Drop-in for the reference tool (filter_split_sets_by_min.c:11-69): each
 * split set with its clusters of fewer than min_members members dropped (none
 * dropped with 0), stored as <prefix>%04d.  Cluster ids are stored as the
 * clusters' positions (the reference stores ids it never sets).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mnhn_dropin.h"

int main(int argc, char** argv) {
  int min_members = 0;
  if (argc < 3) {
    printf("Arguments are: "
           " [int] minimum to consider a cluster \n"
           " [path/prefix] Where to store the filtered splitsets\n "
           " [file1 ... filen] split_sets obtainted from adaptive clustering \n"
           "                   calculations in order from lowest to hight\n");
    return 1;
  }
  sscanf(argv[1], "%i", &min_members);
  const char* prefix = argv[2];
  char* name = (char*)malloc(strlen(prefix) + 16);
  for (int i = 3; i < argc; i++) {
    split_set s = read_split_set(argv[i]);
    if (swgpu_last_dropin_status() != 0) return 1;
    if (min_members) {
      split_set f = filtered_split_set_by_min_size(s, min_members);
      free_split_set_and_associated_clusters(s);
      s = f;
    }
    sprintf(name, "%s%04d", prefix, i - 3);
    store_split_set(name, s);
    free_split_set_and_associated_clusters(s);
  }
  free(name);
  return 0;
}
