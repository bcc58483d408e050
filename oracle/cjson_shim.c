/*
 * Minimal JSON reader exposing the twelve cJSON entry points that the
 * reference's config wrapper calls (include/json_config.hpp in the reference:
 * cJSON_Parse, _Delete, _GetErrorPtr, _GetObjectItemCaseSensitive,
 * _GetArrayItem, _GetArraySize, _IsArray, _IsObject, _IsNumber, _IsBool,
 * _IsTrue, _IsString).
 *
 * TEST INFRASTRUCTURE ONLY: it lets oracle/Makefile link the reference's own
 * CUDA sources into oracle/_ref/main_debug, whose records pin the oracle. The
 * node layout is the public `struct cJSON` declared in the reference's
 * include/cJSON.h (v1.7.19); the parser itself is written here from the JSON
 * grammar (RFC 8259). The prebuilt lib/libcjson.a of the reference is not used.
 */
#include <cJSON.h>

#include <limits.h>
#include <stdlib.h>
#include <string.h>

static const char *g_error = NULL;

typedef struct {
    const char *p;
} cursor;

static void skip_ws(cursor *c) {
    while (*c->p == ' ' || *c->p == '\t' || *c->p == '\n' || *c->p == '\r') c->p++;
}

static cJSON *new_node(int type) {
    cJSON *n = (cJSON *)calloc(1, sizeof(cJSON));
    if (n) n->type = type;
    return n;
}

static cJSON *parse_value(cursor *c, int depth);

static int hexval(char ch) {
    if (ch >= '0' && ch <= '9') return ch - '0';
    if (ch >= 'a' && ch <= 'f') return ch - 'a' + 10;
    if (ch >= 'A' && ch <= 'F') return ch - 'A' + 10;
    return -1;
}

/* Parses a quoted string at c->p; returns a malloc'd UTF-8 copy. */
static char *parse_string_raw(cursor *c) {
    if (*c->p != '"') return NULL;
    const char *s = c->p + 1;
    size_t cap = 16, len = 0;
    char *out = (char *)malloc(cap);
    if (!out) return NULL;
    while (*s && *s != '"') {
        unsigned cp;
        int escaped_unicode = 0;
        if (*s == '\\') {
            s++;
            switch (*s) {
            case '"': cp = '"'; break;
            case '\\': cp = '\\'; break;
            case '/': cp = '/'; break;
            case 'b': cp = '\b'; break;
            case 'f': cp = '\f'; break;
            case 'n': cp = '\n'; break;
            case 'r': cp = '\r'; break;
            case 't': cp = '\t'; break;
            case 'u': {
                cp = 0;
                for (int k = 1; k <= 4; ++k) {
                    int h = hexval(s[k]);
                    if (h < 0) { free(out); return NULL; }
                    cp = cp * 16 + (unsigned)h;
                }
                s += 4;
                escaped_unicode = 1;
                break;
            }
            default: free(out); return NULL;
            }
            s++;
        } else {
            cp = (unsigned char)*s++;
        }
        char enc[4];
        size_t n = 0;
        if (!escaped_unicode || cp < 0x80) {
            /* plain byte (input is already UTF-8) or ASCII escape */
            enc[n++] = (char)cp;
        } else if (cp < 0x800) {
            enc[n++] = (char)(0xC0 | (cp >> 6));
            enc[n++] = (char)(0x80 | (cp & 0x3F));
        } else {
            enc[n++] = (char)(0xE0 | (cp >> 12));
            enc[n++] = (char)(0x80 | ((cp >> 6) & 0x3F));
            enc[n++] = (char)(0x80 | (cp & 0x3F));
        }
        if (len + n + 1 > cap) {
            cap *= 2;
            char *t = (char *)realloc(out, cap);
            if (!t) { free(out); return NULL; }
            out = t;
        }
        memcpy(out + len, enc, n);
        len += n;
    }
    if (*s != '"') { free(out); return NULL; }
    out[len] = '\0';
    c->p = s + 1;
    return out;
}

static cJSON *parse_number(cursor *c) {
    char *end = NULL;
    double v = strtod(c->p, &end);
    if (end == c->p) return NULL;
    cJSON *n = new_node(cJSON_Number);
    if (!n) return NULL;
    n->valuedouble = v;
    if (v >= (double)INT_MAX) n->valueint = INT_MAX;
    else if (v <= (double)INT_MIN) n->valueint = INT_MIN;
    else n->valueint = (int)v;
    c->p = end;
    return n;
}

static void append_child(cJSON *parent, cJSON *item, cJSON **last) {
    if (*last == NULL) {
        parent->child = item;
        item->prev = item; /* cJSON keeps the tail in child->prev */
    } else {
        (*last)->next = item;
        item->prev = *last;
        parent->child->prev = item;
    }
    *last = item;
}

static cJSON *parse_container(cursor *c, int depth, int is_object) {
    cJSON *node = new_node(is_object ? cJSON_Object : cJSON_Array);
    if (!node) return NULL;
    cJSON *last = NULL;
    c->p++; /* '{' or '[' */
    skip_ws(c);
    const char close = is_object ? '}' : ']';
    if (*c->p == close) { c->p++; return node; }
    for (;;) {
        skip_ws(c);
        char *key = NULL;
        if (is_object) {
            key = parse_string_raw(c);
            if (!key) goto fail;
            skip_ws(c);
            if (*c->p != ':') { free(key); goto fail; }
            c->p++;
        }
        cJSON *item = parse_value(c, depth + 1);
        if (!item) { free(key); goto fail; }
        item->string = key;
        append_child(node, item, &last);
        skip_ws(c);
        if (*c->p == ',') { c->p++; continue; }
        if (*c->p == close) { c->p++; return node; }
        goto fail;
    }
fail:
    cJSON_Delete(node);
    return NULL;
}

static cJSON *parse_value(cursor *c, int depth) {
    if (depth > CJSON_NESTING_LIMIT) return NULL;
    skip_ws(c);
    const char ch = *c->p;
    if (ch == '{') return parse_container(c, depth, 1);
    if (ch == '[') return parse_container(c, depth, 0);
    if (ch == '"') {
        char *s = parse_string_raw(c);
        if (!s) return NULL;
        cJSON *n = new_node(cJSON_String);
        if (!n) { free(s); return NULL; }
        n->valuestring = s;
        return n;
    }
    if (strncmp(c->p, "true", 4) == 0) { c->p += 4; cJSON *n = new_node(cJSON_True); if (n) n->valueint = 1; return n; }
    if (strncmp(c->p, "false", 5) == 0) { c->p += 5; return new_node(cJSON_False); }
    if (strncmp(c->p, "null", 4) == 0) { c->p += 4; return new_node(cJSON_NULL); }
    if (ch == '-' || (ch >= '0' && ch <= '9')) return parse_number(c);
    return NULL;
}

CJSON_PUBLIC(cJSON *) cJSON_Parse(const char *value) {
    g_error = NULL;
    if (!value) return NULL;
    cursor c = {value};
    cJSON *root = parse_value(&c, 0);
    if (root) {
        skip_ws(&c);
        if (*c.p == '\0') return root;
        cJSON_Delete(root);
    }
    g_error = c.p;
    return NULL;
}

CJSON_PUBLIC(void) cJSON_Delete(cJSON *item) {
    while (item) {
        cJSON *next = item->next;
        if (item->child) cJSON_Delete(item->child);
        free(item->valuestring);
        free(item->string);
        free(item);
        item = next;
    }
}

CJSON_PUBLIC(const char *) cJSON_GetErrorPtr(void) { return g_error; }

CJSON_PUBLIC(int) cJSON_GetArraySize(const cJSON *array) {
    if (!array) return 0;
    int n = 0;
    for (const cJSON *c = array->child; c; c = c->next) n++;
    return n;
}

CJSON_PUBLIC(cJSON *) cJSON_GetArrayItem(const cJSON *array, int index) {
    if (!array || index < 0) return NULL;
    cJSON *c = array->child;
    while (c && index > 0) { c = c->next; index--; }
    return c;
}

CJSON_PUBLIC(cJSON *) cJSON_GetObjectItemCaseSensitive(const cJSON *const object, const char *const string) {
    if (!object || !string) return NULL;
    for (cJSON *c = object->child; c; c = c->next)
        if (c->string && strcmp(c->string, string) == 0) return c;
    return NULL;
}

CJSON_PUBLIC(cJSON_bool) cJSON_IsArray(const cJSON *const item) { return item && (item->type & 0xFF) == cJSON_Array; }
CJSON_PUBLIC(cJSON_bool) cJSON_IsObject(const cJSON *const item) { return item && (item->type & 0xFF) == cJSON_Object; }
CJSON_PUBLIC(cJSON_bool) cJSON_IsNumber(const cJSON *const item) { return item && (item->type & 0xFF) == cJSON_Number; }
CJSON_PUBLIC(cJSON_bool) cJSON_IsString(const cJSON *const item) { return item && (item->type & 0xFF) == cJSON_String; }
CJSON_PUBLIC(cJSON_bool) cJSON_IsTrue(const cJSON *const item) { return item && (item->type & 0xFF) == cJSON_True; }
CJSON_PUBLIC(cJSON_bool) cJSON_IsBool(const cJSON *const item) {
    return item && (item->type & (cJSON_True | cJSON_False)) != 0;
}
