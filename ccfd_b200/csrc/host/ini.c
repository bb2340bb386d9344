/*
 * .ini parameter parsing with the reference's semantics
 * (src/readInTools.c:38-405):
 *   - a key is every [alnum _] character of the line before the first
 *     '!', '#' or '=', lower-cased;
 *   - the value is every [alnum _ . , -] character after that, up to the
 *     first '!' or '#' (so "(/0.0, 1.0/)" reads as "0.0,1.0");
 *   - reading a key consumes its first occurrence, so repeated keys are
 *     returned in file order;
 *   - integers are read through strtod and truncated, booleans accept
 *     T / True / t / true.
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_host.h"

typedef struct ini_cmd {
	char key[256];
	char value[256];
	int used;
} ini_cmd;

struct ccfd_ini {
	ini_cmd *cmd;
	int n, cap;
};

ccfd_ini *ccfd_ini_parse(const char *text)
{
	ccfd_ini *ini = calloc(1, sizeof(*ini));
	if (!ini)
		return NULL;
	const char *p = text;
	while (p && *p) {
		const char *eol = strchr(p, '\n');
		size_t len = eol ? (size_t)(eol - p) + 1 : strlen(p);
		char key[256], val[256];
		size_t i = 0, j = 0;
		for (; i < len; ++i) {
			unsigned char ch = (unsigned char)p[i];
			if (isalnum(ch) || ch == '_') {
				if (j < sizeof(key) - 1)
					key[j++] = (char)tolower(ch);
			} else if (ch == '!' || ch == '#' || ch == '=') {
				break;
			}
		}
		key[j] = '\0';
		if (j > 0) {
			size_t k = 0;
			for (; i < len; ++i) {
				unsigned char ch = (unsigned char)p[i];
				if (isalnum(ch) || ch == '_' || ch == '.' || ch == ',' || ch == '-') {
					if (k < sizeof(val) - 1)
						val[k++] = (char)ch;
				} else if (ch == '!' || ch == '#') {
					break;
				}
			}
			val[k] = '\0';
			if (ini->n == ini->cap) {
				int cap = ini->cap ? 2 * ini->cap : 64;
				ini_cmd *c = realloc(ini->cmd, sizeof(ini_cmd) * cap);
				if (!c) {
					ccfd_ini_free(ini);
					return NULL;
				}
				ini->cmd = c;
				ini->cap = cap;
			}
			ini_cmd *c = &ini->cmd[ini->n++];
			strcpy(c->key, key);
			strcpy(c->value, val);
			c->used = 0;
		}
		p += len;
	}
	return ini;
}

void ccfd_ini_free(ccfd_ini *ini)
{
	if (!ini)
		return;
	free(ini->cmd);
	free(ini);
}

static void lower_copy(const char *key, char *out, size_t n)
{
	size_t i = 0;
	for (; key[i] && i < n - 1; ++i)
		out[i] = (char)tolower((unsigned char)key[i]);
	out[i] = '\0';
}

/* findCmd: first unused occurrence, consumed; else the default */
static const char *find_cmd(ccfd_ini *ini, const char *key, const char *def)
{
	char lk[256];
	lower_copy(key, lk, sizeof(lk));
	for (int i = 0; i < ini->n; ++i) {
		if (!ini->cmd[i].used && !strcmp(ini->cmd[i].key, lk)) {
			ini->cmd[i].used = 1;
			return ini->cmd[i].value;
		}
	}
	return def;
}

int ccfd_ini_str(ccfd_ini *ini, const char *key, const char *def, char *out, size_t n)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	snprintf(out, n, "%s", v);
	return CCFD_OK;
}

int ccfd_ini_int(ccfd_ini *ini, const char *key, const char *def, long *out)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	*out = (long)strtod(v, NULL);
	return CCFD_OK;
}

int ccfd_ini_dbl(ccfd_ini *ini, const char *key, const char *def, double *out)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	*out = strtod(v, NULL);
	return CCFD_OK;
}

int ccfd_ini_bool(ccfd_ini *ini, const char *key, const char *def, int *out)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	*out = !strcmp(v, "T") || !strcmp(v, "True") || !strcmp(v, "t") ||
	       !strcmp(v, "true");
	return CCFD_OK;
}

/* comma-separated list; a list shorter than n is an error (the reference
 * would dereference a NULL token) */
static int split_list(const char *v, int n, double *out)
{
	char buf[256];
	snprintf(buf, sizeof(buf), "%s", v);
	char *save = NULL;
	char *tok = strtok_r(buf, ",", &save);
	for (int i = 0; i < n; ++i) {
		if (!tok)
			return CCFD_ERR_INI;
		out[i] = strtod(tok, NULL);
		tok = strtok_r(NULL, ",", &save);
	}
	return CCFD_OK;
}

int ccfd_ini_dbl_array(ccfd_ini *ini, const char *key, int n, const char *def, double *out)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	return split_list(v, n, out);
}

int ccfd_ini_int_array(ccfd_ini *ini, const char *key, int n, const char *def, int *out)
{
	const char *v = find_cmd(ini, key, def);
	if (!v)
		return CCFD_ERR_INI;
	double tmp[64];
	if (n > 64)
		return CCFD_ERR_ARG;
	int st = split_list(v, n, tmp);
	for (int i = 0; st == CCFD_OK && i < n; ++i)
		out[i] = (int)tmp[i];
	return st;
}

int ccfd_ini_count(ccfd_ini *ini, const char *key, int proposal, int *out)
{
	char lk[256];
	lower_copy(key, lk, sizeof(lk));
	int count = 0;
	for (int i = 0; i < ini->n; ++i)
		if (!ini->cmd[i].used && !strcmp(ini->cmd[i].key, lk))
			++count;
	if (count == 0) {
		if (proposal == -1)
			return CCFD_ERR_INI;
		*out = proposal;
	} else {
		*out = count;
	}
	return CCFD_OK;
}

int ccfd_ini_remaining(const ccfd_ini *ini)
{
	int r = 0;
	for (int i = 0; i < ini->n; ++i)
		r += !ini->cmd[i].used;
	return r;
}
