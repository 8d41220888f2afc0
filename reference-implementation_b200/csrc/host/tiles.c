/*
 * Tile shape of grouped tensor-core products, per shape class.
 *
 * A grouped launch (tapp_b200_execute_group, the server's grouped units)
 * runs its products' tiles with one of two shapes: 256 x 256 tiles on SM
 * pairs (tile 1: the fewest operand reloads per flop) or 128 x 128 tiles on
 * single SMs (tile 2: four times as many tiles, so small products spread
 * over more SMs and waste less of a tile at their edges). Which is faster
 * depends on the product's shape; the tuner (tapp_b200/tuner.py) times both
 * on synthetic products of each shape class and writes a table that this
 * file reads. Without a table entry a size rule decides.
 *
 * Shape class: (operand mode, floor(log2 M), floor(log2 N), floor(log2 K)),
 * M, N, K the product's GEMM view (rows of A, columns of B, contracted
 * size); batch modes only multiply the tiles. Table file: text, one class
 * per line, "mode m n k tile", '#' starts a comment line. The reference has
 * no counterpart (its batched product is declared only,
 * api/include/tapp/product.h:66-75).
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tb_internal.h"

#define TILE_MAX_ENTRIES 4096

typedef struct {
    int mode, m, n, k, tile;
} tile_entry;

static tile_entry table[TILE_MAX_ENTRIES];
static int n_table;
static pthread_mutex_t table_lock = PTHREAD_MUTEX_INITIALIZER;
static pthread_once_t env_once = PTHREAD_ONCE_INIT;

static int log2_floor(int64_t x)
{
    int b = 0;
    while (x > 1 && b < 62) {
        x >>= 1;
        b++;
    }
    return b;
}

/* reads `path` into the table; returns entries read or -1 */
static int load(const char* path)
{
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    char line[256];
    pthread_mutex_lock(&table_lock);
    n_table = 0;
    while (n_table < TILE_MAX_ENTRIES && fgets(line, sizeof line, f)) {
        tile_entry e;
        if (line[0] == '#' || sscanf(line, "%d %d %d %d %d", &e.mode, &e.m, &e.n, &e.k, &e.tile) != 5) continue;
        if (e.tile == 1 || e.tile == 2) table[n_table++] = e;
    }
    const int n = n_table;
    pthread_mutex_unlock(&table_lock);
    fclose(f);
    return n;
}

static void load_from_env(void)
{
    const char* p = getenv("TAPP_B200_TILE_TABLE");
    if (p && *p) load(p);
}

int tb_tile_choice(const tb_plan* P)
{
    pthread_once(&env_once, load_from_env);
    const int m = log2_floor(P->M.size), n = log2_floor(P->N.size), k = log2_floor(P->K.size);
    int tile = 0;
    pthread_mutex_lock(&table_lock);
    for (int i = 0; i < n_table && !tile; i++)
        if (table[i].mode == P->tc_mode && table[i].m == m && table[i].n == n && table[i].k == k) tile = table[i].tile;
    pthread_mutex_unlock(&table_lock);
    if (tile) return tile;
    /* size rule: SM-pair tiles once a product fills them in both directions */
    return P->M.size >= 256 && P->N.size >= 256 ? 1 : 2;
}

TAPP_error tapp_b200_load_tile_table(const char* path)
{
    pthread_once(&env_once, load_from_env);
    if (!path) {
        pthread_mutex_lock(&table_lock);
        n_table = 0;
        pthread_mutex_unlock(&table_lock);
        return 0;
    }
    return load(path) < 0 ? TAPP_B200_ERR_INVALID : 0;
}
