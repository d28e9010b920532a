/* Gate-list plug-in for bin/qcs: replays the circuit in the text file named
   by QCS_GATELIST. First line: "<num_qubits> <num_clbits>". Then one
   operation per line:
     <gate> <nparams> <p...> <ntargets> <t...> <nnegctrls> <n...> <nctrls> <c...>
     measure <qubit> <clbit>
   Gate names are those of the qcs_simulator_gate_* functions. */
#include <qcs.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
    char name[24];
    int np, nt, nn, nc;
    double p[4];
    bit_num_t t[4], n[8], c[8];
} op_t;

static op_t *ops;
static int nops;
static bit_num_t nq, ncl;

static void fail(const char *msg)
{
    fprintf(stderr, "gatelist: %s\n", msg);
    exit(EXIT_FAILURE);
}

static void read_list(const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f)
        fail("cannot open QCS_GATELIST");
    int a, b;
    if (fscanf(f, "%d %d", &a, &b) != 2)
        fail("bad header");
    nq = (bit_num_t)a;
    ncl = (bit_num_t)b;
    int cap = 1024;
    ops = malloc(sizeof(op_t) * cap);
    char name[24];
    while (fscanf(f, "%23s", name) == 1)
    {
        if (nops == cap)
        {
            cap *= 2;
            ops = realloc(ops, sizeof(op_t) * cap);
        }
        op_t *o = &ops[nops++];
        memset(o, 0, sizeof(*o));
        strcpy(o->name, name);
        int v;
        if (strcmp(name, "measure") == 0)
        {
            if (fscanf(f, "%d %d", &a, &b) != 2)
                fail("bad measure");
            o->t[0] = (bit_num_t)a;
            o->c[0] = (bit_num_t)b;
            continue;
        }
        if (fscanf(f, "%d", &o->np) != 1 || o->np > 4)
            fail("bad parameter count");
        for (int i = 0; i < o->np; ++i)
            if (fscanf(f, "%lf", &o->p[i]) != 1)
                fail("bad parameter");
        if (fscanf(f, "%d", &o->nt) != 1 || o->nt > 4)
            fail("bad target count");
        for (int i = 0; i < o->nt; ++i)
        {
            if (fscanf(f, "%d", &v) != 1)
                fail("bad target");
            o->t[i] = (bit_num_t)v;
        }
        if (fscanf(f, "%d", &o->nn) != 1 || o->nn > 8)
            fail("bad negative control count");
        for (int i = 0; i < o->nn; ++i)
        {
            if (fscanf(f, "%d", &v) != 1)
                fail("bad negative control");
            o->n[i] = (bit_num_t)v;
        }
        if (fscanf(f, "%d", &o->nc) != 1 || o->nc > 8)
            fail("bad control count");
        for (int i = 0; i < o->nc; ++i)
        {
            if (fscanf(f, "%d", &v) != 1)
                fail("bad control");
            o->c[i] = (bit_num_t)v;
        }
    }
    fclose(f);
}

void circuit_init(qcs_simulator *sim)
{
    const char *path = getenv("QCS_GATELIST");
    if (!path)
        fail("set QCS_GATELIST");
    read_list(path);
    qcs_simulator_set_num_qubits(sim, nq);
    qcs_simulator_set_num_clbits(sim, ncl);
}

#define TL o->t, (bit_num_t)o->nt, o->n, (bit_num_t)o->nn, o->c, (bit_num_t)o->nc
#define IS(x) (strcmp(o->name, x) == 0)

void circuit_run(qcs_simulator *sim)
{
    for (int i = 0; i < nops; ++i)
    {
        const op_t *o = &ops[i];
        const double *p = o->p;
        int ok = 1;
        if (IS("measure"))
        {
            bit_t r;
            ok = qcs_simulator_measure_to_clbit(sim, o->t[0], o->c[0], &r);
        }
        else if (IS("global_phase")) ok = qcs_simulator_gate_global_phase(sim, p[0], o->n, (bit_num_t)o->nn, o->c, (bit_num_t)o->nc);
        else if (IS("h")) ok = qcs_simulator_gate_h(sim, TL);
        else if (IS("x")) ok = qcs_simulator_gate_x(sim, TL);
        else if (IS("y")) ok = qcs_simulator_gate_y(sim, TL);
        else if (IS("z")) ok = qcs_simulator_gate_z(sim, TL);
        else if (IS("s")) ok = qcs_simulator_gate_s(sim, TL);
        else if (IS("sdg")) ok = qcs_simulator_gate_sdg(sim, TL);
        else if (IS("t")) ok = qcs_simulator_gate_t(sim, TL);
        else if (IS("tdg")) ok = qcs_simulator_gate_tdg(sim, TL);
        else if (IS("sx")) ok = qcs_simulator_gate_sx(sim, TL);
        else if (IS("sxdg")) ok = qcs_simulator_gate_sxdg(sim, TL);
        else if (IS("id")) ok = qcs_simulator_gate_id(sim, TL);
        else if (IS("rx")) ok = qcs_simulator_gate_rx(sim, p[0], TL);
        else if (IS("ry")) ok = qcs_simulator_gate_ry(sim, p[0], TL);
        else if (IS("rz")) ok = qcs_simulator_gate_rz(sim, p[0], TL);
        else if (IS("u1")) ok = qcs_simulator_gate_u1(sim, p[0], TL);
        else if (IS("p")) ok = qcs_simulator_gate_p(sim, p[0], TL);
        else if (IS("u2")) ok = qcs_simulator_gate_u2(sim, p[0], p[1], TL);
        else if (IS("r")) ok = qcs_simulator_gate_r(sim, p[0], p[1], TL);
        else if (IS("u3")) ok = qcs_simulator_gate_u3(sim, p[0], p[1], p[2], TL);
        else if (IS("u")) ok = qcs_simulator_gate_u(sim, p[0], p[1], p[2], TL);
        else if (IS("u4")) ok = qcs_simulator_gate_u4(sim, p[0], p[1], p[2], p[3], TL);
        else if (IS("swap")) ok = qcs_simulator_gate_swap(sim, TL);
        else if (IS("iswap")) ok = qcs_simulator_gate_iswap(sim, TL);
        else if (IS("dcx")) ok = qcs_simulator_gate_dcx(sim, TL);
        else if (IS("ecr")) ok = qcs_simulator_gate_ecr(sim, TL);
        else if (IS("rxx")) ok = qcs_simulator_gate_rxx(sim, p[0], TL);
        else if (IS("ryy")) ok = qcs_simulator_gate_ryy(sim, p[0], TL);
        else if (IS("rzz")) ok = qcs_simulator_gate_rzz(sim, p[0], TL);
        else if (IS("rzx")) ok = qcs_simulator_gate_rzx(sim, p[0], TL);
        else if (IS("xx_plus_yy")) ok = qcs_simulator_gate_xx_plus_yy(sim, p[0], p[1], TL);
        else if (IS("xx_minus_yy")) ok = qcs_simulator_gate_xx_minus_yy(sim, p[0], p[1], TL);
        else if (IS("rccx")) ok = qcs_simulator_gate_rccx(sim, TL);
        else if (IS("rcccx")) ok = qcs_simulator_gate_rcccx(sim, TL);
        else fail("unknown gate");
        if (!ok)
            fail("a gate call failed");
    }
}
