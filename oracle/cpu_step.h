/*
 * cpu_step.h — oracle restatement of `Cpu::step` (src/cpu.rs:245-1146).
 *
 * TEST INFRASTRUCTURE ONLY: this file is part of the CPU oracle that the
 * parity tests, the smoke check and the CPU baseline use as the checker.
 * Nothing in the product path includes it.
 *
 * It is included once per memory type.  Before including, define:
 *   STEP_FN         name of the generated function
 *   MEM_T           memory type
 *   MREAD(m, a)     one bus read  (uint16_t a) -> uint8_t
 *   MWRITE(m, a, v) one bus write
 *   PHANTOM_READ(m, a)      a read whose value the reference discards
 *   RMW_OLD_WRITE(m, a, v)  read-modify-write's write of the original value
 * The bus operations are issued in exactly the order of the reference,
 * including every phantom read and the read-modify-write double write,
 * because phantom accesses have side effects on the Atari bus (bank
 * hotspots, INTIM's underflow flag, GRP0/GRP1 shadow registers).
 *
 * Returns the instruction's cycle count, or 0 for an illegal opcode (the
 * reference panics there, src/cpu.rs:1139-1141); in that case pc has already
 * advanced past the opcode and cpu->cycles is unchanged.
 */

static uint8_t STEP_FN(orc_cpu* c, MEM_T* m)
{
    uint8_t cyc = 1;
    uint8_t op = MREAD(m, c->pc);                     /* cycle 1: opcode */
    c->pc = (uint16_t)(c->pc + 1);

    switch (op) {
    /* NOP (cpu.rs:257-261) */
    case 0xEA:
        PHANTOM_READ(m, c->pc); cyc++;
        break;

    /* flag ops (cpu.rs:266-280) */
    case 0x18: case 0x38: case 0x58: case 0x78: case 0xB8: case 0xD8: case 0xF8:
        PHANTOM_READ(m, c->pc); cyc++;
        switch (op) {
        case 0x18: orc_setf(c, F_C, 0); break;
        case 0x38: orc_setf(c, F_C, 1); break;
        case 0x58: orc_setf(c, F_I, 0); break;
        case 0x78: orc_setf(c, F_I, 1); break;
        case 0xB8: orc_setf(c, F_V, 0); break;
        case 0xD8: orc_setf(c, F_D, 0); break;
        default:   orc_setf(c, F_D, 1); break;
        }
        break;

    /* register transfers (cpu.rs:285-298) */
    case 0xAA: case 0xA8: case 0x8A: case 0x98: case 0xBA: case 0x9A:
        PHANTOM_READ(m, c->pc); cyc++;
        switch (op) {
        case 0xAA: c->x = c->a; orc_zn(c, c->x); break;
        case 0xA8: c->y = c->a; orc_zn(c, c->y); break;
        case 0x8A: c->a = c->x; orc_zn(c, c->a); break;
        case 0x98: c->a = c->y; orc_zn(c, c->a); break;
        case 0xBA: c->x = c->sp; orc_zn(c, c->x); break;
        default:   c->sp = c->x; break;                  /* TXS: no flags */
        }
        break;

    /* INX/INY/DEX/DEY (cpu.rs:303-314) */
    case 0xE8: case 0xC8: case 0xCA: case 0x88:
        PHANTOM_READ(m, c->pc); cyc++;
        switch (op) {
        case 0xE8: c->x++; orc_zn(c, c->x); break;
        case 0xC8: c->y++; orc_zn(c, c->y); break;
        case 0xCA: c->x--; orc_zn(c, c->x); break;
        default:   c->y--; orc_zn(c, c->y); break;
        }
        break;

    /* shifts on A (cpu.rs:319-330) */
    case 0x0A: case 0x4A: case 0x2A: case 0x6A:
        PHANTOM_READ(m, c->pc); cyc++;
        switch (op) {
        case 0x0A: c->a = orc_asl(c, c->a); break;
        case 0x4A: c->a = orc_lsr(c, c->a); break;
        case 0x2A: c->a = orc_rol(c, c->a); break;
        default:   c->a = orc_ror(c, c->a); break;
        }
        break;

    /* immediate (cpu.rs:336-356) */
    case 0x69: case 0x29: case 0xC9: case 0xE0: case 0xC0: case 0x49: case 0xA9:
    case 0xA2: case 0xA0: case 0x09: case 0xE9: {
        uint8_t v = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* zero page read (cpu.rs:362-391) */
    case 0xA5: case 0xA6: case 0xA4: case 0x65: case 0x25: case 0xC5: case 0xE4:
    case 0xC4: case 0x45: case 0x05: case 0xE5: case 0x24: {
        uint16_t ad = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint8_t v = MREAD(m, ad); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* zero page write (cpu.rs:396-410) */
    case 0x85: case 0x86: case 0x84: {
        uint16_t ad = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        MWRITE(m, ad, orc_store_val(c, op)); cyc++;
        break;
    }

    /* zp,X read (cpu.rs:415-438) */
    case 0xB5: case 0xB4: case 0x75: case 0x35: case 0xD5: case 0x55: case 0x15: case 0xF5: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        uint8_t v = MREAD(m, (uint8_t)(base + c->x)); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* zp,X write (cpu.rs:443-460) */
    case 0x95: case 0x94: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        MWRITE(m, (uint8_t)(base + c->x), orc_store_val(c, op)); cyc++;
        break;
    }

    /* zp,Y read: LDX (cpu.rs:465-479) */
    case 0xB6: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        uint8_t v = MREAD(m, (uint8_t)(base + c->y)); cyc++;
        c->x = v; orc_zn(c, c->x);
        break;
    }

    /* zp,Y write: STX (cpu.rs:484-493) */
    case 0x96: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        MWRITE(m, (uint8_t)(base + c->y), c->x); cyc++;
        break;
    }

    /* zp RMW (cpu.rs:498-521) */
    case 0x06: case 0x46: case 0x26: case 0x66: case 0xE6: case 0xC6: {
        uint16_t ad = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint8_t v = MREAD(m, ad); cyc++;
        RMW_OLD_WRITE(m, ad, v); cyc++;
        MWRITE(m, ad, orc_rmw(c, op, v)); cyc++;
        break;
    }

    /* zp,X RMW (cpu.rs:526-553) */
    case 0x16: case 0x56: case 0x36: case 0x76: case 0xF6: case 0xD6: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        uint16_t ad = (uint8_t)(base + c->x);
        uint8_t v = MREAD(m, ad); cyc++;
        RMW_OLD_WRITE(m, ad, v); cyc++;
        MWRITE(m, ad, orc_rmw(c, op, v)); cyc++;
        break;
    }

    /* absolute read (cpu.rs:559-592) */
    case 0xAD: case 0xAE: case 0xAC: case 0x6D: case 0x2D: case 0xCD: case 0xEC:
    case 0xCC: case 0x4D: case 0x0D: case 0xED: case 0x2C: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint8_t v = MREAD(m, (uint16_t)((hi << 8) | lo)); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* absolute write (cpu.rs:597-613) */
    case 0x8D: case 0x8E: case 0x8C: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        MWRITE(m, (uint16_t)((hi << 8) | lo), orc_store_val(c, op)); cyc++;
        break;
    }

    /* absolute RMW (cpu.rs:618-644) */
    case 0x0E: case 0x4E: case 0x2E: case 0x6E: case 0xEE: case 0xCE: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t ad = (uint16_t)((hi << 8) | lo);
        uint8_t v = MREAD(m, ad); cyc++;
        RMW_OLD_WRITE(m, ad, v); cyc++;
        MWRITE(m, ad, orc_rmw(c, op, v)); cyc++;
        break;
    }

    /* abs,X / abs,Y read with page-cross phantom (cpu.rs:649-679, 741-769) */
    case 0xBD: case 0xBC: case 0x7D: case 0x3D: case 0xDD: case 0x5D: case 0x1D: case 0xFD:
    case 0xB9: case 0xBE: case 0x79: case 0x39: case 0xD9: case 0x59: case 0x19: case 0xF9: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t base = (uint16_t)((hi << 8) | lo);
        uint8_t idx = ((op & 0x1C) == 0x1C && op != 0xBE) ? c->x : c->y;
        uint16_t eff = (uint16_t)(base + idx);
        if ((base & 0xFF00) != (eff & 0xFF00)) {
            PHANTOM_READ(m, (uint16_t)((base & 0xFF00) | (eff & 0x00FF))); cyc++;
        }
        uint8_t v = MREAD(m, eff); cyc++;
        if (op == 0xBE) { c->x = v; orc_zn(c, c->x); }
        else orc_read_op(c, op, v);
        break;
    }

    /* STA abs,X / abs,Y: fixup read always (cpu.rs:684-700, 774-788) */
    case 0x9D: case 0x99: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t base = (uint16_t)((hi << 8) | lo);
        uint16_t eff = (uint16_t)(base + (op == 0x9D ? c->x : c->y));
        PHANTOM_READ(m, (uint16_t)((base & 0xFF00) | (eff & 0x00FF))); cyc++;
        MWRITE(m, eff, c->a); cyc++;
        break;
    }

    /* abs,X RMW (cpu.rs:705-736) */
    case 0x1E: case 0x5E: case 0x3E: case 0x7E: case 0xFE: case 0xDE: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t base = (uint16_t)((hi << 8) | lo);
        uint16_t eff = (uint16_t)(base + c->x);
        PHANTOM_READ(m, (uint16_t)((base & 0xFF00) | (eff & 0x00FF))); cyc++;
        uint8_t v = MREAD(m, eff); cyc++;
        RMW_OLD_WRITE(m, eff, v); cyc++;
        MWRITE(m, eff, orc_rmw(c, op, v)); cyc++;
        break;
    }

    /* (zp,X) read (cpu.rs:793-822) */
    case 0xA1: case 0x61: case 0x21: case 0xC1: case 0x41: case 0x01: case 0xE1: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        uint8_t ptr = (uint8_t)(base + c->x);
        uint16_t lo = MREAD(m, ptr); cyc++;
        uint16_t hi = MREAD(m, (uint8_t)(ptr + 1)); cyc++;
        uint8_t v = MREAD(m, (uint16_t)((hi << 8) | lo)); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* STA (zp,X) (cpu.rs:827-841) */
    case 0x81: {
        uint8_t base = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, base); cyc++;
        uint8_t ptr = (uint8_t)(base + c->x);
        uint16_t lo = MREAD(m, ptr); cyc++;
        uint16_t hi = MREAD(m, (uint8_t)(ptr + 1)); cyc++;
        MWRITE(m, (uint16_t)((hi << 8) | lo), c->a); cyc++;
        break;
    }

    /* (zp),Y read (cpu.rs:846-879) */
    case 0xB1: case 0x71: case 0x31: case 0xD1: case 0x51: case 0x11: case 0xF1: {
        uint8_t zp = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t lo = MREAD(m, zp); cyc++;
        uint16_t hi = MREAD(m, (uint8_t)(zp + 1)); cyc++;
        uint16_t base = (uint16_t)((hi << 8) | lo);
        uint16_t eff = (uint16_t)(base + c->y);
        if ((base & 0xFF00) != (eff & 0xFF00)) {
            PHANTOM_READ(m, (uint16_t)((base & 0xFF00) | (eff & 0x00FF))); cyc++;
        }
        uint8_t v = MREAD(m, eff); cyc++;
        orc_read_op(c, op, v);
        break;
    }

    /* STA (zp),Y (cpu.rs:884-901) */
    case 0x91: {
        uint8_t zp = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t lo = MREAD(m, zp); cyc++;
        uint16_t hi = MREAD(m, (uint8_t)(zp + 1)); cyc++;
        uint16_t base = (uint16_t)((hi << 8) | lo);
        uint16_t eff = (uint16_t)(base + c->y);
        PHANTOM_READ(m, (uint16_t)((base & 0xFF00) | (eff & 0x00FF))); cyc++;
        MWRITE(m, eff, c->a); cyc++;
        break;
    }

    /* branches (cpu.rs:906-944) */
    case 0x90: case 0xB0: case 0xF0: case 0x30: case 0xD0: case 0x10: case 0x50: case 0x70: {
        int8_t off = (int8_t)MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        int taken;
        switch (op) {
        case 0x90: taken = !(c->p & F_C); break;
        case 0xB0: taken = (c->p & F_C) != 0; break;
        case 0xF0: taken = (c->p & F_Z) != 0; break;
        case 0x30: taken = (c->p & F_N) != 0; break;
        case 0xD0: taken = !(c->p & F_Z); break;
        case 0x10: taken = !(c->p & F_N); break;
        case 0x50: taken = !(c->p & F_V); break;
        default:   taken = (c->p & F_V) != 0; break;
        }
        if (taken) {
            PHANTOM_READ(m, c->pc); cyc++;
            uint16_t old = c->pc;
            uint16_t npc = (uint16_t)(c->pc + (uint16_t)(int16_t)off);
            if ((old & 0xFF00) != (npc & 0xFF00)) {
                PHANTOM_READ(m, (uint16_t)((old & 0xFF00) | (npc & 0x00FF))); cyc++;
            }
            c->pc = npc;
        }
        break;
    }

    /* JMP abs (cpu.rs:949-956): pc is not advanced past the high byte */
    case 0x4C: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); cyc++;
        c->pc = (uint16_t)((hi << 8) | lo);
        break;
    }

    /* JMP (ind) with the page-wrap bug (cpu.rs:961-978) */
    case 0x6C: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t hi = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        uint16_t ptr = (uint16_t)((hi << 8) | lo);
        uint16_t tlo = MREAD(m, ptr); cyc++;
        uint16_t thi = MREAD(m, (uint16_t)((ptr & 0xFF00) | ((uint16_t)(ptr + 1) & 0x00FF))); cyc++;
        c->pc = (uint16_t)((thi << 8) | tlo);
        break;
    }

    /* JSR (cpu.rs:983-1005) */
    case 0x20: {
        uint16_t lo = MREAD(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        PHANTOM_READ(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        uint16_t ret = c->pc;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), (uint8_t)(ret >> 8)); c->sp--; cyc++;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), (uint8_t)ret); c->sp--; cyc++;
        uint16_t hi = MREAD(m, c->pc); cyc++;
        c->pc = (uint16_t)((hi << 8) | lo);
        break;
    }

    /* RTS (cpu.rs:1010-1028) */
    case 0x60: {
        PHANTOM_READ(m, c->pc); cyc++;
        PHANTOM_READ(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->sp++; uint16_t lo = MREAD(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->sp++; uint16_t hi = MREAD(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        uint16_t ra = (uint16_t)((hi << 8) | lo);
        PHANTOM_READ(m, ra); cyc++;
        c->pc = (uint16_t)(ra + 1);
        break;
    }

    /* RTI (cpu.rs:1033-1051) */
    case 0x40: {
        PHANTOM_READ(m, c->pc); cyc++;
        PHANTOM_READ(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->sp++; c->p = (uint8_t)(MREAD(m, (uint16_t)(0x0100 | c->sp)) & ~(F_B | F_U)); cyc++;
        c->sp++; uint16_t lo = MREAD(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->sp++; uint16_t hi = MREAD(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->pc = (uint16_t)((hi << 8) | lo);
        break;
    }

    /* BRK (cpu.rs:1056-1080) */
    case 0x00: {
        PHANTOM_READ(m, c->pc); c->pc = (uint16_t)(c->pc + 1); cyc++;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), (uint8_t)(c->pc >> 8)); c->sp--; cyc++;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), (uint8_t)c->pc); c->sp--; cyc++;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), (uint8_t)(c->p | F_B | F_U)); c->sp--; cyc++;
        orc_setf(c, F_I, 1);
        uint16_t lo = MREAD(m, 0xFFFE); cyc++;
        uint16_t hi = MREAD(m, 0xFFFF); cyc++;
        c->pc = (uint16_t)((hi << 8) | lo);
        break;
    }

    /* PHA / PHP (cpu.rs:1085-1105) */
    case 0x48: case 0x08:
        PHANTOM_READ(m, c->pc); cyc++;
        MWRITE(m, (uint16_t)(0x0100 | c->sp), op == 0x48 ? c->a : (uint8_t)(c->p | F_B | F_U));
        c->sp--; cyc++;
        break;

    /* PLA / PLP (cpu.rs:1110-1137) */
    case 0x68: case 0x28: {
        PHANTOM_READ(m, c->pc); cyc++;
        PHANTOM_READ(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        c->sp++; uint8_t v = MREAD(m, (uint16_t)(0x0100 | c->sp)); cyc++;
        if (op == 0x68) { c->a = v; orc_zn(c, c->a); }
        else c->p = (uint8_t)(v & ~(F_B | F_U));
        break;
    }

    default:
        return 0;   /* illegal opcode */
    }

    c->cycles += cyc;
    return cyc;
}
