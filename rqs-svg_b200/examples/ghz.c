/* GHZ plug-in for bin/qcs: H on qubit 0, CX from 0 to every other qubit,
   measure every qubit into the clbit of the same index. The width comes from
   the NUM_QUBITS environment variable. Every shot prints all-0 or all-1. */
#include <qcs.h>
#include <stdio.h>
#include <stdlib.h>

static bit_num_t width;

void circuit_init(qcs_simulator *sim)
{
    const char *s = getenv("NUM_QUBITS");
    width = (bit_num_t)(s ? atoi(s) : 0);
    if (width <= 0)
    {
        fprintf(stderr, "set NUM_QUBITS to a positive qubit count\n");
        exit(EXIT_FAILURE);
    }
    qcs_simulator_set_num_qubits(sim, width);
    qcs_simulator_set_num_clbits(sim, width);
}

void circuit_run(qcs_simulator *sim)
{
    bit_num_t zero = 0;
    qcs_simulator_gate_h(sim, &zero, 1, NULL, 0, NULL, 0);
    for (bit_num_t q = 1; q < width; ++q)
        qcs_simulator_gate_x(sim, &q, 1, NULL, 0, &zero, 1);
    for (bit_num_t q = 0; q < width; ++q)
    {
        bit_t r;
        qcs_simulator_measure_to_clbit(sim, q, q, &r);
    }
}
